// StateVectorB200.hpp — C++ host API mirroring lightning.qubit's state-vector classes,
// implemented on the C ABI of libb200sv (include/b200sv.h) only.
//
// Reference interfaces kept (paths relative to pennylane_lightning/core/src):
//   StateVectorBase::applyOperation / applyOperations / applyGenerator / applyMatrix
//     simulators/base/StateVectorBase.hpp:99-194
//   StateVectorLQubitManaged(num_qubits), (data, length) constructors
//     simulators/lightning_qubit/StateVectorLQubitManaged.hpp:72-129
//   PL_ABORT / LightningException error convention  utils/Error.hpp:22-63
//
// The amplitudes live in device memory; getDataVector() / updateData() move
// them between host and device explicitly.
#pragma once

#include <b200sv.h>

#include <complex>
#include <cstdint>
#include <exception>
#include <span>
#include <string>
#include <unordered_map>
#include <vector>

namespace Pennylane::LightningB200 {

// Same role as Pennylane::Util::LightningException (utils/Error.hpp:22-63).
class LightningException : public std::exception {
    std::string msg_;

  public:
    explicit LightningException(std::string msg) : msg_(std::move(msg)) {}
    [[nodiscard]] const char *what() const noexcept override { return msg_.c_str(); }
};

inline void check(int status) {
    if (status != B200SV_OK) throw LightningException(b200sv_last_error());
}

// Gate / generator name tables: CS/gates/Constant.hpp:46-140.
inline const std::unordered_map<std::string, uint32_t> &gate_ids() {
    static const std::unordered_map<std::string, uint32_t> m = {
        {"Identity", 0}, {"PauliX", 1}, {"PauliY", 2}, {"PauliZ", 3}, {"Hadamard", 4}, {"S", 5}, {"T", 6},
        {"PhaseShift", 7}, {"RX", 8}, {"RY", 9}, {"RZ", 10}, {"Rot", 11}, {"CNOT", 12}, {"CY", 13}, {"CZ", 14},
        {"SWAP", 15}, {"IsingXX", 16}, {"IsingXY", 17}, {"IsingYY", 18}, {"IsingZZ", 19},
        {"ControlledPhaseShift", 20}, {"CRX", 21}, {"CRY", 22}, {"CRZ", 23}, {"CRot", 24},
        {"SingleExcitation", 25}, {"SingleExcitationMinus", 26}, {"SingleExcitationPlus", 27},
        {"Toffoli", 28}, {"CSWAP", 29}, {"DoubleExcitation", 30}, {"DoubleExcitationMinus", 31},
        {"DoubleExcitationPlus", 32}, {"MultiRZ", 33}};
    return m;
}
inline const std::vector<std::string> &gate_names() {
    static const std::vector<std::string> v = [] {
        std::vector<std::string> r(34);
        for (auto &[k, id] : gate_ids()) r[id] = k;
        return r;
    }();
    return v;
}
inline const std::unordered_map<std::string, uint32_t> &generator_ids() {
    static const std::unordered_map<std::string, uint32_t> m = {
        {"PhaseShift", 0}, {"RX", 1}, {"RY", 2}, {"RZ", 3}, {"IsingXX", 4}, {"IsingXY", 5}, {"IsingYY", 6},
        {"IsingZZ", 7}, {"CRX", 8}, {"CRY", 9}, {"CRZ", 10}, {"ControlledPhaseShift", 11},
        {"SingleExcitation", 12}, {"SingleExcitationMinus", 13}, {"SingleExcitationPlus", 14},
        {"DoubleExcitation", 15}, {"DoubleExcitationMinus", 16}, {"DoubleExcitationPlus", 17}, {"MultiRZ", 18}};
    return m;
}
inline uint32_t lookup_gate(const std::string &name) {
    // The dispatcher's error for an unknown operation (DynamicDispatcher.hpp:322-326).
    auto it = gate_ids().find(name);
    if (it == gate_ids().end()) throw LightningException("Cannot find a registered kernel for a given gate: " + name);
    return it->second;
}
inline uint32_t op_id(const std::string &name) {
    if (name == "QubitStateVector" || name == "BasisState" || name == "StatePrep") return B200SV_OP_SKIP;
    if (name == "QubitUnitary" || name == "Matrix") return B200SV_OP_MATRIX;
    return lookup_gate(name);
}

template <class T> class StateVectorB200 {
  public:
    using PrecisionT = T;
    using ComplexT = std::complex<PrecisionT>;
    static constexpr int dtype = sizeof(PrecisionT) == 4 ? B200SV_C64 : B200SV_C128;

    explicit StateVectorB200(size_t num_qubits) : nq_(num_qubits) { check(b200sv_create((uint32_t)nq_, dtype, &h_)); }
    StateVectorB200(const ComplexT *data, size_t length) : nq_(log2_exact(length)) {
        check(b200sv_create((uint32_t)nq_, dtype, &h_));
        updateData(data, length);
    }
    StateVectorB200(const StateVectorB200 &o) : nq_(o.nq_) {
        check(b200sv_create((uint32_t)nq_, dtype, &h_));
        check(b200sv_copy(h_, o.h_));
    }
    StateVectorB200 &operator=(const StateVectorB200 &) = delete;
    StateVectorB200(StateVectorB200 &&o) noexcept : nq_(o.nq_), h_(o.h_) { o.h_ = nullptr; }
    ~StateVectorB200() {
        if (h_) b200sv_destroy(h_);
    }

    [[nodiscard]] size_t getNumQubits() const { return nq_; }
    [[nodiscard]] size_t getLength() const { return size_t(1) << nq_; }
    [[nodiscard]] b200sv_handle handle() const { return h_; }

    void updateData(const ComplexT *data, size_t length) {
        if (length != getLength()) throw LightningException("The length of the data must equal 2^num_qubits");
        check(b200sv_upload(h_, data, length));
    }
    void getData(ComplexT *out, size_t length) const {
        if (length != getLength()) throw LightningException("The length of the buffer must equal 2^num_qubits");
        check(b200sv_download(h_, out, length));
    }
    [[nodiscard]] std::vector<ComplexT> getDataVector() const {
        std::vector<ComplexT> v(getLength());
        getData(v.data(), v.size());
        return v;
    }
    void resetStateVector() { check(b200sv_set_basis_state(h_, 0)); }
    void setBasisState(size_t index) { check(b200sv_set_basis_state(h_, index)); }

    // StateVectorBase.hpp:99-105
    void applyOperation(const std::string &opName, const std::vector<size_t> &wires, bool inverse = false,
                        const std::vector<PrecisionT> &params = {}) {
        const uint32_t id = lookup_gate(opName);
        std::vector<uint32_t> w(wires.begin(), wires.end());
        std::vector<double> p(params.begin(), params.end());
        check(b200sv_apply_gate(h_, id, w.data(), (uint32_t)w.size(), inverse ? 1 : 0, p.data(), (uint32_t)p.size()));
    }
    // StateVectorBase.hpp:117-165
    void applyOperations(const std::vector<std::string> &ops, const std::vector<std::vector<size_t>> &wires,
                         const std::vector<bool> &inverse, const std::vector<std::vector<PrecisionT>> &params) {
        const size_t n = ops.size();
        if (wires.size() != n || inverse.size() != n || params.size() != n)
            throw LightningException("Invalid arguments: number of operations, wires, inverses, and parameters "
                                     "must all be equal");
        for (size_t i = 0; i < n; ++i) applyOperation(ops[i], wires[i], inverse[i], params[i]);
    }
    void applyOperations(const std::vector<std::string> &ops, const std::vector<std::vector<size_t>> &wires,
                         const std::vector<bool> &inverse) {
        const size_t n = ops.size();
        if (wires.size() != n || inverse.size() != n)
            throw LightningException("Invalid arguments: number of operations, wires, and inverses must all be equal");
        for (size_t i = 0; i < n; ++i) applyOperation(ops[i], wires[i], inverse[i], {});
    }
    // StateVectorBase.hpp:174-179
    PrecisionT applyGenerator(const std::string &opName, const std::vector<size_t> &wires, bool adj = false) {
        auto it = generator_ids().find(opName);
        if (it == generator_ids().end())
            throw LightningException("Cannot find a registered kernel for a given generator: " + opName);
        std::vector<uint32_t> w(wires.begin(), wires.end());
        double s = 0;
        check(b200sv_apply_generator(h_, it->second, w.data(), (uint32_t)w.size(), adj ? 1 : 0, &s));
        return (PrecisionT)s;
    }
    // StateVectorBase.hpp:189-194 and LQ/StateVectorLQubit.hpp:329-365
    void applyMatrix(const ComplexT *matrix, const std::vector<size_t> &wires, bool inverse = false) {
        if (wires.empty()) throw LightningException("Number of wires must be larger than 0");
        std::vector<uint32_t> w(wires.begin(), wires.end());
        check(b200sv_apply_matrix(h_, matrix, w.data(), (uint32_t)w.size(), inverse ? 1 : 0));
    }
    void applyMatrix(const std::vector<ComplexT> &matrix, const std::vector<size_t> &wires, bool inverse = false) {
        if (matrix.size() != (size_t(1) << (2 * wires.size())))
            throw LightningException("The size of matrix does not match with the given number of wires");
        applyMatrix(matrix.data(), wires, inverse);
    }

  private:
    static size_t log2_exact(size_t len) {
        size_t n = 0;
        while ((size_t(1) << n) < len) ++n;
        if ((size_t(1) << n) != len || len < 2) throw LightningException("The length of the data must be a power of 2");
        return n;
    }
    size_t nq_;
    b200sv_handle h_ = nullptr;
};

}  // namespace Pennylane::LightningB200
