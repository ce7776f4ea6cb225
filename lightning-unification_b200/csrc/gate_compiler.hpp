// gate_compiler.hpp — host-side translation of lightning.qubit operations into
// the five kernel forms of libb200sv.
//
// The reference dispatches every (gate, kernel) pair to its own loop
// (LQ/gates/DynamicDispatcher.hpp:316-352 → GateImplementationsLM.hpp:390-1352).
// Here a gate becomes one of five forms, each a single coalesced pass:
//   Dense  — 2^k x 2^k matrix on k target bits, optionally gated by control bits
//   Diag   — 2^k phases on k target bits (k <= 2), optionally gated by controls
//   Swap   — exchange of two amplitudes of each group (X, CNOT, SWAP, Toffoli, CSWAP)
//   Pair   — 2x2 block on two rows of a 2^k group, the other rows scaled by gamma
//            (single / double excitations and their generators)
//   Parity — phase chosen by the parity of selected bits (MultiRZ)
// Coefficients (cos, sin, exp) are computed here in FP64 with the reference's
// formulas, so the device needs no transcendental functions.
#pragma once

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace b200sv {

using cd = std::complex<double>;

struct ArgError : std::invalid_argument {
    using std::invalid_argument::invalid_argument;
};
struct Unsupported : std::runtime_error {
    using std::runtime_error::runtime_error;
};

enum class Kind : int { Noop = 0, Dense, Diag, Swap, Pair, Parity };

struct GateDesc {
    Kind kind = Kind::Noop;
    int k = 0;                    // number of target ("matrix") bits
    std::vector<uint32_t> tbits;  // target bit positions; tbits[0] is the matrix-index MSB
    std::vector<uint32_t> cbits;  // control bit positions (amplitudes with all of them set)
    std::vector<cd> m;            // Dense: 4^k row-major; Diag: 2^k phases
    uint32_t sa = 0, sb = 0;      // Swap: exchanged rows
    uint32_t pa = 0, pb = 0;      // Pair: rows of the 2x2 block
    cd m2[4] = {};                // Pair: block (row-major over (pa, pb))
    cd gamma{1.0, 0.0};           // Pair: factor on the other rows
    uint64_t pmask = 0;           // Parity: selected bits
    cd pphase[2] = {};            // Parity: phase for even / odd parity
};

// Gate metadata: CS/gates/Constant.hpp:46-269 (names, wire counts, parameter counts).
struct GateInfo {
    const char *name;
    int nwires;   // -1: any (MultiRZ)
    int nparams;
};
inline const GateInfo *gate_table() {
    static const GateInfo t[] = {
        {"Identity", 1, 0},          {"PauliX", 1, 0},
        {"PauliY", 1, 0},            {"PauliZ", 1, 0},
        {"Hadamard", 1, 0},          {"S", 1, 0},
        {"T", 1, 0},                 {"PhaseShift", 1, 1},
        {"RX", 1, 1},                {"RY", 1, 1},
        {"RZ", 1, 1},                {"Rot", 1, 3},
        {"CNOT", 2, 0},              {"CY", 2, 0},
        {"CZ", 2, 0},                {"SWAP", 2, 0},
        {"IsingXX", 2, 1},           {"IsingXY", 2, 1},
        {"IsingYY", 2, 1},           {"IsingZZ", 2, 1},
        {"ControlledPhaseShift", 2, 1}, {"CRX", 2, 1},
        {"CRY", 2, 1},               {"CRZ", 2, 1},
        {"CRot", 2, 3},              {"SingleExcitation", 2, 1},
        {"SingleExcitationMinus", 2, 1}, {"SingleExcitationPlus", 2, 1},
        {"Toffoli", 3, 0},           {"CSWAP", 3, 0},
        {"DoubleExcitation", 4, 1},  {"DoubleExcitationMinus", 4, 1},
        {"DoubleExcitationPlus", 4, 1}, {"MultiRZ", -1, 1},
    };
    return t;
}
constexpr uint32_t kNumGates = 34;

// Generator names: CS/gates/Constant.hpp:102-140; ids CS/gates/GateOperation.hpp:75-98.
inline const char *generator_name(uint32_t g) {
    static const char *n[] = {"PhaseShift", "RX", "RY", "RZ", "IsingXX", "IsingXY", "IsingYY",
                              "IsingZZ", "CRX", "CRY", "CRZ", "ControlledPhaseShift",
                              "SingleExcitation", "SingleExcitationMinus",
                              "SingleExcitationPlus", "DoubleExcitation",
                              "DoubleExcitationMinus", "DoubleExcitationPlus", "MultiRZ"};
    return g < 19 ? n[g] : "?";
}
constexpr uint32_t kNumGenerators = 19;

inline int generator_wires(uint32_t g) {
    static const int w[] = {1, 1, 1, 1, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 4, 4, 4, -1};
    return w[g];
}

// Gate id -> generator id (the gates the adjoint method differentiates), or -1.
inline int generator_of_gate(uint32_t gate) {
    switch (gate) {
    case 7: return 0;    // PhaseShift
    case 8: return 1;    // RX
    case 9: return 2;    // RY
    case 10: return 3;   // RZ
    case 16: return 4;   // IsingXX
    case 17: return 5;   // IsingXY
    case 18: return 6;   // IsingYY
    case 19: return 7;   // IsingZZ
    case 21: return 8;   // CRX
    case 22: return 9;   // CRY
    case 23: return 10;  // CRZ
    case 20: return 11;  // ControlledPhaseShift
    case 25: return 12;  // SingleExcitation
    case 26: return 13;  // SingleExcitationMinus
    case 27: return 14;  // SingleExcitationPlus
    case 30: return 15;  // DoubleExcitation
    case 31: return 16;  // DoubleExcitationMinus
    case 32: return 17;  // DoubleExcitationPlus
    case 33: return 18;  // MultiRZ
    default: return -1;
    }
}

inline void check_wires(const uint32_t *wires, uint32_t nwires, uint32_t nq, const char *what) {
    for (uint32_t i = 0; i < nwires; ++i) {
        if (wires[i] >= nq)
            throw ArgError(std::string(what) + ": wire " + std::to_string(wires[i]) +
                           " out of range for " + std::to_string(nq) + " qubits");
        for (uint32_t j = 0; j < i; ++j)
            if (wires[i] == wires[j])
                throw ArgError(std::string(what) + ": wires must be distinct");
    }
}

inline uint32_t bitpos(uint32_t wire, uint32_t nq) { return nq - 1 - wire; }

inline cd expi(double a) { return {std::cos(a), std::sin(a)}; }

// conjugate transpose of a row-major d x d matrix
inline std::vector<cd> dagger(const std::vector<cd> &m, size_t d) {
    std::vector<cd> r(d * d);
    for (size_t i = 0; i < d; ++i)
        for (size_t j = 0; j < d; ++j) r[j * d + i] = std::conj(m[i * d + j]);
    return r;
}

inline GateDesc dense(std::vector<uint32_t> tb, std::vector<uint32_t> cb, std::vector<cd> m) {
    GateDesc g;
    g.kind = Kind::Dense;
    g.k = (int)tb.size();
    g.tbits = std::move(tb);
    g.cbits = std::move(cb);
    g.m = std::move(m);
    return g;
}
inline GateDesc diag(std::vector<uint32_t> tb, std::vector<uint32_t> cb, std::vector<cd> ph) {
    GateDesc g;
    g.kind = Kind::Diag;
    g.k = (int)tb.size();
    g.tbits = std::move(tb);
    g.cbits = std::move(cb);
    g.m = std::move(ph);
    return g;
}
inline GateDesc swapg(std::vector<uint32_t> tb, std::vector<uint32_t> cb, uint32_t a, uint32_t b) {
    GateDesc g;
    g.kind = Kind::Swap;
    g.k = (int)tb.size();
    g.tbits = std::move(tb);
    g.cbits = std::move(cb);
    g.sa = a;
    g.sb = b;
    return g;
}
inline GateDesc pairg(std::vector<uint32_t> tb, uint32_t a, uint32_t b, cd m00, cd m01, cd m10,
                      cd m11, cd gamma) {
    GateDesc g;
    g.kind = Kind::Pair;
    g.k = (int)tb.size();
    g.tbits = std::move(tb);
    g.pa = a;
    g.pb = b;
    g.m2[0] = m00; g.m2[1] = m01; g.m2[2] = m10; g.m2[3] = m11;
    g.gamma = gamma;
    return g;
}

// RZ · RY · RZ product of CS/gates/Gates.hpp:340-364 (getRot).
inline std::vector<cd> rot_matrix(double phi, double theta, double omega) {
    const double c = std::cos(theta / 2), s = std::sin(theta / 2);
    const double p = phi + omega, m = phi - omega;
    return {cd(std::cos(p / 2) * c, -std::sin(p / 2) * c), cd(-std::cos(m / 2) * s, -std::sin(m / 2) * s),
            cd(std::cos(m / 2) * s, -std::sin(m / 2) * s), cd(std::cos(p / 2) * c, std::sin(p / 2) * c)};
}

// Compile applyOperation(gate, wires, inverse, params) for an nq-qubit state.
// Formulas follow GateImplementationsLM.hpp:390-1352 and GateImplementationsLM.cpp.
inline GateDesc compile_gate(uint32_t gate, const uint32_t *wires, uint32_t nwires, bool inv,
                             const double *params, uint32_t nparams, uint32_t nq) {
    if (gate >= kNumGates) throw ArgError("applyOperation: unknown gate id " + std::to_string(gate));
    const GateInfo &gi = gate_table()[gate];
    if (gi.nwires >= 0 && (int)nwires != gi.nwires)
        throw ArgError(std::string(gi.name) + ": expected " + std::to_string(gi.nwires) +
                       " wires, got " + std::to_string(nwires));
    if (gi.nwires < 0 && nwires == 0) throw ArgError(std::string(gi.name) + ": needs at least one wire");
    if ((int)nparams != gi.nparams)
        throw ArgError(std::string(gi.name) + ": expected " + std::to_string(gi.nparams) +
                       " parameters, got " + std::to_string(nparams));
    check_wires(wires, nwires, nq, gi.name);
    std::vector<uint32_t> b(nwires);
    for (uint32_t i = 0; i < nwires; ++i) b[i] = bitpos(wires[i], nq);
    const double th = nparams ? params[0] : 0.0;
    const double c = std::cos(th / 2), s = std::sin(th / 2);
    const double sg = inv ? -1.0 : 1.0;
    const cd I(0, 1);
    const double h = 0.70710678118654752440;  // 1/sqrt(2)
    switch (gate) {
    case 0: return GateDesc{};  // Identity
    case 1: return swapg({b[0]}, {}, 0, 1);
    case 2: return dense({b[0]}, {}, {0.0, -I, I, 0.0});
    case 3: return diag({}, {b[0]}, {-1.0});
    case 4: return dense({b[0]}, {}, {h, h, h, -h});
    case 5: return diag({}, {b[0]}, {inv ? -I : I});
    case 6: return diag({}, {b[0]}, {cd(h, inv ? -h : h)});
    case 7: return diag({}, {b[0]}, {expi(sg * th)});
    case 8: return dense({b[0]}, {}, {c, -I * (sg * s), -I * (sg * s), c});
    case 9: return dense({b[0]}, {}, {c, -sg * s, sg * s, c});
    case 10: return diag({b[0]}, {}, {cd(c, -sg * s), cd(c, sg * s)});
    case 11: {
        auto m = rot_matrix(params[0], params[1], params[2]);
        return dense({b[0]}, {}, inv ? dagger(m, 2) : m);
    }
    case 12: return swapg({b[1]}, {b[0]}, 0, 1);
    case 13: return dense({b[1]}, {b[0]}, {0.0, -I, I, 0.0});
    case 14: return diag({}, {b[0], b[1]}, {-1.0});
    case 15: return swapg({b[0], b[1]}, {}, 1, 2);
    case 16: {  // IsingXX: c I - i s X⊗X
        const cd a = -I * (sg * s);
        return dense({b[0], b[1]}, {}, {c, 0, 0, a, 0, c, a, 0, 0, a, c, 0, a, 0, 0, c});
    }
    case 17: {  // IsingXY: identity on |00>,|11>; c, +i s coupling |01>,|10>
        const cd a = I * (sg * s);
        return dense({b[0], b[1]}, {}, {1, 0, 0, 0, 0, c, a, 0, 0, a, c, 0, 0, 0, 0, 1});
    }
    case 18: {  // IsingYY
        const cd a = I * (sg * s);
        return dense({b[0], b[1]}, {}, {c, 0, 0, a, 0, c, -a, 0, 0, -a, c, 0, a, 0, 0, c});
    }
    case 19: {
        const cd f(c, -sg * s), e(c, sg * s);
        return diag({b[0], b[1]}, {}, {f, e, e, f});
    }
    case 20: return diag({}, {b[0], b[1]}, {expi(sg * th)});
    case 21: return dense({b[1]}, {b[0]}, {c, -I * (sg * s), -I * (sg * s), c});
    case 22: return dense({b[1]}, {b[0]}, {c, -sg * s, sg * s, c});
    case 23: return diag({b[1]}, {b[0]}, {cd(c, -sg * s), cd(c, sg * s)});
    case 24: {
        auto m = rot_matrix(params[0], params[1], params[2]);
        return dense({b[1]}, {b[0]}, inv ? dagger(m, 2) : m);
    }
    case 25: return pairg({b[0], b[1]}, 1, 2, c, -sg * s, sg * s, c, 1.0);
    case 26: return pairg({b[0], b[1]}, 1, 2, c, -sg * s, sg * s, c, expi(-sg * th / 2));
    case 27: return pairg({b[0], b[1]}, 1, 2, c, -sg * s, sg * s, c, expi(sg * th / 2));
    case 28: return swapg({b[2]}, {b[0], b[1]}, 0, 1);
    case 29: return swapg({b[1], b[2]}, {b[0]}, 1, 2);
    case 30: return pairg({b[0], b[1], b[2], b[3]}, 3, 12, c, -sg * s, sg * s, c, 1.0);
    case 31: return pairg({b[0], b[1], b[2], b[3]}, 3, 12, c, -sg * s, sg * s, c, expi(-sg * th / 2));
    case 32: return pairg({b[0], b[1], b[2], b[3]}, 3, 12, c, -sg * s, sg * s, c, expi(sg * th / 2));
    case 33: {
        GateDesc g;
        g.kind = Kind::Parity;
        for (auto x : b) g.pmask |= (uint64_t(1) << x);
        g.pphase[0] = cd(c, -sg * s);
        g.pphase[1] = cd(c, sg * s);
        return g;
    }
    }
    throw ArgError("applyOperation: unhandled gate");
}

// applyMatrix (LQ/StateVectorLQubit.hpp:329-365): row-major 4^k, wires[0] = MSB.
inline GateDesc compile_matrix(const cd *mat, const uint32_t *wires, uint32_t nwires, bool inv,
                               uint32_t nq) {
    if (nwires == 0) throw ArgError("applyMatrix: number of wires must be larger than 0");
    check_wires(wires, nwires, nq, "applyMatrix");
    const size_t d = size_t(1) << nwires;
    std::vector<cd> m(mat, mat + d * d);
    std::vector<uint32_t> b(nwires);
    for (uint32_t i = 0; i < nwires; ++i) b[i] = bitpos(wires[i], nq);
    return dense(b, {}, inv ? dagger(m, d) : m);
}

// applyGenerator: the generator G as an operator on its wires plus the scale of
// GateImplementationsLM.hpp:1355-1639, PauliGenerator.hpp:34-56 and
// GateImplementationsPI.cpp:129-204.  Every form here acts on whole groups (no
// control bits), so the same descriptor also drives the fused <bra|G|ket> kernel.
inline GateDesc compile_generator(uint32_t gen, const uint32_t *wires, uint32_t nwires, uint32_t nq,
                                  double *scale) {
    if (gen >= kNumGenerators) throw ArgError("applyGenerator: unknown generator id " + std::to_string(gen));
    const int nw = generator_wires(gen);
    if (nw >= 0 && (int)nwires != nw)
        throw ArgError(std::string("Generator") + generator_name(gen) + ": expected " +
                       std::to_string(nw) + " wires");
    if (nwires == 0) throw ArgError("applyGenerator: needs at least one wire");
    check_wires(wires, nwires, nq, "applyGenerator");
    std::vector<uint32_t> b(nwires);
    for (uint32_t i = 0; i < nwires; ++i) b[i] = bitpos(wires[i], nq);
    const cd I(0, 1);
    switch (gen) {
    case 0: *scale = 1.0; return diag({b[0]}, {}, {0.0, 1.0});
    case 1: *scale = -0.5; return pairg({b[0]}, 0, 1, 0.0, 1.0, 1.0, 0.0, 1.0);
    case 2: *scale = -0.5; return pairg({b[0]}, 0, 1, 0.0, -I, I, 0.0, 1.0);
    case 3: *scale = -0.5; return diag({b[0]}, {}, {1.0, -1.0});
    case 4: *scale = -0.5;
        return dense({b[0], b[1]}, {}, {0, 0, 0, 1, 0, 0, 1, 0, 0, 1, 0, 0, 1, 0, 0, 0});
    case 5: *scale = 0.5;
        return dense({b[0], b[1]}, {}, {0, 0, 0, 0, 0, 0, 1, 0, 0, 1, 0, 0, 0, 0, 0, 0});
    case 6: *scale = -0.5;
        return dense({b[0], b[1]}, {}, {0, 0, 0, -1, 0, 0, 1, 0, 0, 1, 0, 0, -1, 0, 0, 0});
    case 7: *scale = -0.5; return diag({b[0], b[1]}, {}, {1.0, -1.0, -1.0, 1.0});
    case 8: *scale = -0.5;
        return dense({b[0], b[1]}, {}, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 1, 0});
    case 9: *scale = -0.5;
        return dense({b[0], b[1]}, {}, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -I, 0, 0, I, 0});
    case 10: *scale = -0.5; return diag({b[0], b[1]}, {}, {0.0, 0.0, 1.0, -1.0});
    case 11: *scale = 1.0; return diag({b[0], b[1]}, {}, {0.0, 0.0, 0.0, 1.0});
    case 12: *scale = -0.5; return pairg({b[0], b[1]}, 1, 2, 0.0, -I, I, 0.0, 0.0);
    case 13: *scale = -0.5; return pairg({b[0], b[1]}, 1, 2, 0.0, -I, I, 0.0, 1.0);
    case 14: *scale = -0.5; return pairg({b[0], b[1]}, 1, 2, 0.0, -I, I, 0.0, -1.0);
    case 15: *scale = -0.5; return pairg({b[0], b[1], b[2], b[3]}, 3, 12, 0.0, -I, I, 0.0, 0.0);
    case 16: *scale = -0.5; return pairg({b[0], b[1], b[2], b[3]}, 3, 12, 0.0, -I, I, 0.0, 1.0);
    case 17: *scale = -0.5; return pairg({b[0], b[1], b[2], b[3]}, 3, 12, 0.0, -I, I, 0.0, -1.0);
    case 18: {
        *scale = -0.5;
        GateDesc g;
        g.kind = Kind::Parity;
        for (auto x : b) g.pmask |= (uint64_t(1) << x);
        g.pphase[0] = 1.0;
        g.pphase[1] = -1.0;
        return g;
    }
    }
    throw ArgError("applyGenerator: unhandled generator");
}

}  // namespace b200sv
