// sv_capi.cu — extern "C" entry points of libb200sv (declared in include/b200sv.h).
//
// Host orchestration of the plain form: one state per handle, one gate per
// launch, all work stream-ordered on the handle's stream; results are read back
// only where the ABI returns host data.
#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/b200sv.h"
#include "sv_internal.hpp"

using namespace b200sv;

struct b200sv_state {
    uint32_t nq = 0;
    int dtype = B200SV_C128;
    int device = 0;
    cudaStream_t own = nullptr;
    cudaStream_t ext = nullptr;
    bool has_ext = false;          // set_stream called: ext (NULL = legacy default stream)
    void *d_state = nullptr;
    double *d_partials = nullptr;  // kPartialsCapacity doubles, then the arrival counter
    unsigned int *arrival() const { return reinterpret_cast<unsigned int *>(d_partials + kPartialsCapacity); }
    double *d_small = nullptr;     // small results (kSmall doubles)
    double *h_small = nullptr;     // pinned mirror of d_small
    void *d_matrix = nullptr;      // dense matrix staging
    size_t matrix_bytes = 0;
    void *d_scratch[2] = {nullptr, nullptr};  // two state-sized work buffers (lazy)
    void *h_stage[2] = {nullptr, nullptr};    // pinned staging halves for host-array uploads (lazy)
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};
    cudaStream_t stream() const { return has_ext ? ext : own; }
    size_t amp_bytes() const { return dtype == B200SV_C64 ? 8 : 16; }
    size_t state_bytes() const { return amp_bytes() << nq; }
};

namespace {

constexpr size_t kSmall = 4096;
thread_local std::string g_last_error;

template <class F> int guard(F &&f) {
    try {
        g_last_error.clear();
        f();
        return B200SV_OK;
    } catch (const ArgError &e) {
        g_last_error = e.what();
        return B200SV_ERR_ARGUMENT;
    } catch (const Unsupported &e) {
        g_last_error = e.what();
        return B200SV_ERR_UNSUPPORTED;
    } catch (const AllocError &e) {
        g_last_error = e.what();
        return B200SV_ERR_ALLOC;
    } catch (const CudaError &e) {
        g_last_error = e.what();
        return B200SV_ERR_CUDA;
    } catch (const std::bad_alloc &) {
        g_last_error = "host allocation failed";
        return B200SV_ERR_ALLOC;
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return B200SV_ERR_ARGUMENT;
    }
}

void need(bool ok, const char *msg) {
    if (!ok) throw ArgError(msg);
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) B200SV_CUDA(cudaSetDevice(dev));
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

void ensure_matrix(b200sv_state *h, size_t bytes) {
    if (bytes <= h->matrix_bytes) return;
    if (h->d_matrix) {
        B200SV_CUDA(cudaStreamSynchronize(h->stream()));
        B200SV_CUDA(cudaFree(h->d_matrix));
        h->d_matrix = nullptr;
        h->matrix_bytes = 0;
    }
    size_t want = std::max<size_t>(bytes, 64 * 16 * 64);
    B200SV_CUDA(cudaMalloc(&h->d_matrix, want));
    h->matrix_bytes = want;
}

void *scratch(b200sv_state *h, int i) {
    if (!h->d_scratch[i]) B200SV_CUDA(cudaMalloc(&h->d_scratch[i], h->state_bytes()));
    return h->d_scratch[i];
}

void apply_desc(b200sv_state *h, void *const *states, int nstates, const GateDesc &g) {
    if (g.kind == Kind::Dense && g.k >= 3) {
        size_t need_b = g.k >= 4 ? h->amp_bytes() * g.m.size() : 0;
        if (h->dtype == B200SV_C64 && dense_tc_applies(h->nq, g)) need_b = std::max(need_b, dense_tc_scratch_bytes(g.k));
        if (need_b) ensure_matrix(h, need_b);
    }
    if (h->dtype == B200SV_C64) launch_gate<float>(states, nstates, h->nq, g, h->d_matrix, h->stream());
    else launch_gate<double>(states, nstates, h->nq, g, h->d_matrix, h->stream());
}

void apply_desc_multi(b200sv_state *h, const std::vector<void *> &states, const GateDesc &g) {
    for (size_t i = 0; i < states.size(); i += kMaxStatesPerLaunch) {
        const int cnt = (int)std::min<size_t>(kMaxStatesPerLaunch, states.size() - i);
        apply_desc(h, states.data() + i, cnt, g);
    }
}

std::vector<cd> read_matrix(const void *m, size_t count, int dtype) {
    std::vector<cd> r(count);
    if (dtype == B200SV_C64) {
        const float *f = static_cast<const float *>(m);
        for (size_t i = 0; i < count; ++i) r[i] = cd(f[2 * i], f[2 * i + 1]);
    } else {
        const double *d = static_cast<const double *>(m);
        for (size_t i = 0; i < count; ++i) r[i] = cd(d[2 * i], d[2 * i + 1]);
    }
    return r;
}

// ---- operations ------------------------------------------------------------
struct OpRec {
    uint32_t gate;
    std::vector<uint32_t> wires;
    bool inverse;
    std::vector<double> params;
    std::vector<cd> matrix;
};

std::vector<OpRec> read_ops(const b200sv_op *ops, uint32_t nops, int dtype) {
    need(nops == 0 || ops != nullptr, "operations pointer is NULL");
    std::vector<OpRec> r(nops);
    for (uint32_t i = 0; i < nops; ++i) {
        const b200sv_op &o = ops[i];
        need(o.nwires == 0 || o.wires, "operation wires pointer is NULL");
        need(o.nparams == 0 || o.params, "operation params pointer is NULL");
        r[i].gate = o.gate;
        r[i].wires.assign(o.wires, o.wires + o.nwires);
        r[i].inverse = o.inverse != 0;
        r[i].params.assign(o.params, o.params + o.nparams);
        if (o.gate == B200SV_OP_MATRIX) {
            need(o.matrix != nullptr, "matrix operation without matrix");
            need(o.nwires > 0 && o.nwires <= 11, "matrix operation needs 1..11 wires");
            const size_t d = size_t(1) << o.nwires;
            r[i].matrix = read_matrix(o.matrix, d * d, dtype);
        }
    }
    return r;
}

GateDesc compile_op(const OpRec &o, bool inverse, uint32_t nq) {
    if (o.gate == B200SV_OP_SKIP) return GateDesc{};
    if (o.gate == B200SV_OP_MATRIX)
        return compile_matrix(o.matrix.data(), o.wires.data(), (uint32_t)o.wires.size(), inverse, nq);
    return compile_gate(o.gate, o.wires.data(), (uint32_t)o.wires.size(), inverse, o.params.data(),
                        (uint32_t)o.params.size(), nq);
}

// ---- observables ---------------------------------------------------------------
struct FactorRec {
    bool named;
    uint32_t gate;
    std::vector<uint32_t> wires;
    std::vector<cd> matrix;
};
struct TermRec {
    double coeff;
    std::vector<FactorRec> f;
    bool is_pauli = false;
    PauliWord word;
};
struct ObsRec {
    std::vector<TermRec> terms;
    bool all_pauli() const {
        for (auto &t : terms)
            if (!t.is_pauli) return false;
        return true;
    }
};

ObsRec read_obs(const b200sv_observable &o, uint32_t nq, int dtype) {
    ObsRec r;
    need(o.nterms == 0 || o.terms, "observable terms pointer is NULL");
    for (uint32_t t = 0; t < o.nterms; ++t) {
        const b200sv_term &bt = o.terms[t];
        need(bt.nfactors == 0 || bt.factors, "observable factors pointer is NULL");
        TermRec tr;
        tr.coeff = bt.coeff;
        tr.is_pauli = true;
        std::vector<uint32_t> seen;
        for (uint32_t f = 0; f < bt.nfactors; ++f) {
            const b200sv_factor &bf = bt.factors[f];
            need(bf.nwires == 0 || bf.wires, "observable wires pointer is NULL");
            FactorRec fr;
            fr.named = bf.kind == B200SV_FACTOR_NAMED;
            fr.gate = bf.gate;
            fr.wires.assign(bf.wires, bf.wires + bf.nwires);
            check_wires(fr.wires.data(), (uint32_t)fr.wires.size(), nq, "observable");
            for (auto w : fr.wires) {
                if (std::find(seen.begin(), seen.end(), w) != seen.end())
                    throw ArgError("All wires in observables must be disjoint.");
                seen.push_back(w);
            }
            if (!fr.named) {
                need(bf.matrix != nullptr, "Hermitian observable without matrix");
                need(bf.nwires > 0 && bf.nwires <= 11, "Hermitian observable needs 1..11 wires");
                const size_t d = size_t(1) << bf.nwires;
                fr.matrix = read_matrix(bf.matrix, d * d, dtype);
                tr.is_pauli = false;
            } else {
                need(fr.gate < kNumGates, "unknown observable name");
                const bool pauli = fr.gate <= 3 && fr.wires.size() == 1;
                if (!pauli) tr.is_pauli = false;
                if (pauli) {
                    const uint64_t bit = uint64_t(1) << bitpos(fr.wires[0], nq);
                    if (fr.gate == 1) tr.word.xmask |= bit;
                    if (fr.gate == 2) {
                        tr.word.xmask |= bit;
                        tr.word.zmask |= bit;
                        tr.word.ny++;
                    }
                    if (fr.gate == 3) tr.word.zmask |= bit;
                }
            }
            tr.f.push_back(std::move(fr));
        }
        r.terms.push_back(std::move(tr));
    }
    return r;
}

void apply_factor(b200sv_state *h, void *state, const FactorRec &f) {
    GateDesc g = f.named ? compile_gate(f.gate, f.wires.data(), (uint32_t)f.wires.size(), false, nullptr, 0, h->nq)
                         : compile_matrix(f.matrix.data(), f.wires.data(), (uint32_t)f.wires.size(), false, h->nq);
    void *s[1] = {state};
    apply_desc(h, s, 1, g);
}

// out = O psi (observable applied out of place); tmp is a second work buffer
void apply_observable(b200sv_state *h, const ObsRec &o, const void *psi, void *out, void *tmp) {
    const cudaStream_t st = h->stream();
    const bool single = o.terms.size() == 1 && o.terms[0].coeff == 1.0;
    if (single) {
        B200SV_CUDA(cudaMemcpyAsync(out, psi, h->state_bytes(), cudaMemcpyDeviceToDevice, st));
        for (auto &f : o.terms[0].f) apply_factor(h, out, f);
        return;
    }
    B200SV_CUDA(cudaMemsetAsync(out, 0, h->state_bytes(), st));
    for (auto &t : o.terms) {
        if (t.is_pauli) {
            if (h->dtype == B200SV_C64) axpy_pauli<float>(out, psi, h->nq, t.word, t.coeff, st);
            else axpy_pauli<double>(out, psi, h->nq, t.word, t.coeff, st);
        } else {
            B200SV_CUDA(cudaMemcpyAsync(tmp, psi, h->state_bytes(), cudaMemcpyDeviceToDevice, st));
            for (auto &f : t.f) apply_factor(h, tmp, f);
            if (h->dtype == B200SV_C64) axpy<float>(out, tmp, h->nq, t.coeff, st);
            else axpy<double>(out, tmp, h->nq, t.coeff, st);
        }
    }
}

// per-term Pauli values of an all-Pauli observable (host vector, term order).  Words sorted by
// X mask.  Diagonal words (two or more, 12+ qubits) share Walsh-Hadamard passes of
// reduce_pauli_diag, up to 256 per pass.  The other words are packed, first fit in X-mask
// order, into tiles of 12 or 13 bits (pauli_tile_bits): a tile holding two or more distinct X
// masks is one
// tiled pass of reduce_pauli_tiled (up to 32 words).  The rest: words whose X mask stays below
// 4 MiB of amplitudes share passes of reduce_pauli_multi, up to 32 per pass, their partner
// amplitudes coming from L2; each wider X mask gets pair passes of reduce_pauli_group, where a
// thread reads both amplitudes of a pair.  The state crosses HBM once per pass in every kind.
std::vector<double> pauli_term_values(b200sv_state *h, const void *psi, const std::vector<PauliWord> &words) {
    const cudaStream_t st = h->stream();
    std::vector<double> vals(words.size(), 0.0);
    std::vector<size_t> order(words.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return words[a].xmask < words[b].xmask; });
    const uint64_t near = (uint64_t(4) << 20) / h->amp_bytes();  // partner distance kept in L2
    enum Kind { DIAG, MULTI, PAIR, TILED };
    struct Pass {
        size_t begin, count;  // into seq
        Kind kind;
    };
    std::vector<size_t> seq;  // word indices, each pass's words contiguous
    seq.reserve(words.size());
    std::vector<Pass> passes;
    size_t i = 0;
    // diagonal words (sorted first): Walsh-Hadamard passes, any number of words per read
    size_t ndiag = 0;
    while (ndiag < order.size() && words[order[ndiag]].xmask == 0) ++ndiag;
    if (h->nq >= 12 && ndiag >= 2) {
        for (size_t d = 0; d < ndiag; d += 256) {
            passes.push_back(Pass{seq.size(), std::min<size_t>(256, ndiag - d), DIAG});
            for (size_t q = d; q < d + passes.back().count; ++q) seq.push_back(order[q]);
        }
        i = ndiag;
    }
    // tiles: first fit of the distinct X masks (chunks of <= 32 words) in ascending order
    struct Tile {
        uint64_t xunion;
        int nmasks;
        std::vector<size_t> w;  // positions in order
    };
    std::vector<Tile> tiles;
    std::vector<size_t> rest;  // positions in order left to the multi and pair passes
    for (size_t r = i; r < order.size();) {
        const uint64_t m = words[order[r]].xmask;
        size_t e = r;
        while (e < order.size() && words[order[e]].xmask == m) ++e;
        for (size_t c = r; c < e; c += 32) {
            const size_t n = std::min<size_t>(32, e - c);
            Tile *t = nullptr;
            if (m != 0 && pauli_tile_bits(m, h->nq, h->amp_bytes())) {
                for (auto &tl : tiles)
                    if (tl.w.size() + n <= 32 && pauli_tile_bits(tl.xunion | m, h->nq, h->amp_bytes())) {
                        t = &tl;
                        break;
                    }
                if (!t) {
                    tiles.push_back(Tile{0, 0, {}});
                    t = &tiles.back();
                }
            }
            if (!t) {
                for (size_t q = c; q < c + n; ++q) rest.push_back(q);
                continue;
            }
            const bool fresh = t->w.empty() || words[order[t->w.back()]].xmask != m;
            t->xunion |= m;
            t->nmasks += fresh;
            for (size_t q = c; q < c + n; ++q) t->w.push_back(q);
        }
        r = e;
    }
    for (auto &tl : tiles) {
        if (tl.nmasks < 2) {
            rest.insert(rest.end(), tl.w.begin(), tl.w.end());
            continue;
        }
        passes.push_back(Pass{seq.size(), tl.w.size(), TILED});
        for (size_t q : tl.w) seq.push_back(order[q]);
    }
    std::sort(rest.begin(), rest.end());  // X-mask order
    size_t k = 0;
    while (k < rest.size() && words[order[rest[k]]].xmask < near) {
        // up to 32 words and 8 distinct X masks per pass: each mask adds a partner read per
        // amplitude, so wider passes cost as much as pair passes
        size_t c = 0;
        int masks = 0;
        while (k + c < rest.size() && c < 32 && words[order[rest[k + c]]].xmask < near) {
            const uint64_t m = words[order[rest[k + c]]].xmask;
            const bool fresh = c == 0 || m != words[order[rest[k + c - 1]]].xmask;
            if (fresh && m != 0 && masks == 8) break;
            if (fresh && m != 0) ++masks;
            ++c;
        }
        passes.push_back(Pass{seq.size(), c, MULTI});
        for (size_t q = k; q < k + c; ++q) seq.push_back(order[rest[q]]);
        k += c;
    }
    while (k < rest.size()) {
        size_t c = 1;
        while (k + c < rest.size() && c < 32 && words[order[rest[k + c]]].xmask == words[order[rest[k]]].xmask) ++c;
        passes.push_back(Pass{seq.size(), c, PAIR});
        for (size_t q = k; q < k + c; ++q) seq.push_back(order[rest[q]]);
        k += c;
    }
    const bool c64 = h->dtype == B200SV_C64;
    size_t pi = 0;
    while (pi < passes.size()) {
        size_t batch = 0;
        const size_t first = passes[pi].begin;
        while (pi < passes.size() && batch + passes[pi].count <= kSmall) {
            const Pass &ps = passes[pi];
            std::vector<PauliWord> grp;
            for (size_t q = 0; q < ps.count; ++q) grp.push_back(words[seq[ps.begin + q]]);
            const int cnt = (int)ps.count;
            double *out = h->d_small + batch;
            switch (ps.kind) {
            case DIAG: {
                // the Z masks ride at the end of the partials buffer, past what the pass uses
                std::vector<uint64_t> zm(ps.count);
                for (size_t q = 0; q < ps.count; ++q) zm[q] = grp[q].zmask;
                uint64_t *dz = reinterpret_cast<uint64_t *>(h->d_partials + kPartialsCapacity - 256);
                B200SV_CUDA(cudaMemcpyAsync(dz, zm.data(), zm.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
                if (c64) reduce_pauli_diag<float>(psi, h->nq, dz, cnt, h->d_partials, kPartialsCapacity - 256, out, st);
                else reduce_pauli_diag<double>(psi, h->nq, dz, cnt, h->d_partials, kPartialsCapacity - 256, out, st);
                break;
            }
            case TILED:
                if (c64) reduce_pauli_tiled<float>(psi, h->nq, grp.data(), cnt, h->d_partials, out, st);
                else reduce_pauli_tiled<double>(psi, h->nq, grp.data(), cnt, h->d_partials, out, st);
                break;
            case MULTI:
                if (c64) reduce_pauli_multi<float>(psi, h->nq, grp.data(), cnt, h->d_partials, out, st);
                else reduce_pauli_multi<double>(psi, h->nq, grp.data(), cnt, h->d_partials, out, st);
                break;
            case PAIR:
                if (c64) reduce_pauli_group<float>(psi, h->nq, grp.data(), cnt, h->d_partials, out, st);
                else reduce_pauli_group<double>(psi, h->nq, grp.data(), cnt, h->d_partials, out, st);
                break;
            }
            batch += ps.count;
            ++pi;
        }
        B200SV_CUDA(cudaMemcpyAsync(h->h_small, h->d_small, batch * sizeof(double), cudaMemcpyDeviceToHost, st));
        B200SV_CUDA(cudaStreamSynchronize(st));
        for (size_t q = 0; q < batch; ++q) vals[seq[first + q]] = h->h_small[q];
    }
    return vals;
}

double read_small(b200sv_state *h, size_t i) {
    B200SV_CUDA(cudaMemcpyAsync(h->h_small, h->d_small, (i + 1) * sizeof(double), cudaMemcpyDeviceToHost, h->stream()));
    B200SV_CUDA(cudaStreamSynchronize(h->stream()));
    return h->h_small[i];
}

double norm2_of(b200sv_state *h, const void *a) {
    if (h->dtype == B200SV_C64) reduce_norm2<float>(a, h->nq, h->d_partials, h->d_small, h->stream());
    else reduce_norm2<double>(a, h->nq, h->d_partials, h->d_small, h->stream());
    return read_small(h, 0);
}

void inner_of(b200sv_state *h, const void *bra, const void *ket, double *re, double *im) {
    if (h->dtype == B200SV_C64) reduce_inner<float>(bra, ket, h->nq, h->d_partials, h->d_small, h->stream());
    else reduce_inner<double>(bra, ket, h->nq, h->d_partials, h->d_small, h->stream());
    read_small(h, 1);
    *re = h->h_small[0];
    *im = h->h_small[1];
}

double expval_impl(b200sv_state *h, const ObsRec &o) {
    if (o.terms.empty()) return 0.0;
    if (o.all_pauli()) {
        std::vector<PauliWord> words;
        for (auto &t : o.terms) words.push_back(t.word);
        auto v = pauli_term_values(h, h->d_state, words);
        double s = 0.0;
        for (size_t i = 0; i < v.size(); ++i) s += o.terms[i].coeff * v[i];
        return s;
    }
    if (o.terms.size() == 1 && o.terms[0].f.size() == 1 && !o.terms[0].f[0].named &&
        o.terms[0].f[0].wires.size() <= 4) {
        const FactorRec &f = o.terms[0].f[0];
        GateDesc g = compile_matrix(f.matrix.data(), f.wires.data(), (uint32_t)f.wires.size(), false, h->nq);
        ensure_matrix(h, h->amp_bytes() * g.m.size());
        if (h->dtype == B200SV_C64)
            reduce_dense_expval<float>(h->d_state, h->nq, g, h->d_matrix, h->d_partials, h->d_small, h->stream());
        else
            reduce_dense_expval<double>(h->d_state, h->nq, g, h->d_matrix, h->d_partials, h->d_small, h->stream());
        return o.terms[0].coeff * read_small(h, 0);
    }
    void *out = scratch(h, 0);
    void *tmp = o.terms.size() > 1 ? scratch(h, 1) : nullptr;
    apply_observable(h, o, h->d_state, out, tmp);
    double re, im;
    inner_of(h, h->d_state, out, &re, &im);
    return re;
}

double var_impl(b200sv_state *h, const ObsRec &o) {
    if (o.terms.size() == 1 && o.terms[0].is_pauli) {
        // <P^2> = <psi|psi> for a Pauli word: one pass gives <P> and the norm
        const double c = o.terms[0].coeff;
        if (h->dtype == B200SV_C64)
            reduce_pauli_group<float>(h->d_state, h->nq, &o.terms[0].word, 1, h->d_partials, h->d_small, h->stream(), true);
        else
            reduce_pauli_group<double>(h->d_state, h->nq, &o.terms[0].word, 1, h->d_partials, h->d_small, h->stream(), true);
        read_small(h, 1);
        const double ev = h->h_small[0], n2 = h->h_small[1];
        return c * c * n2 - (c * ev) * (c * ev);
    }
    void *out = scratch(h, 0);
    void *tmp = o.terms.size() > 1 ? scratch(h, 1) : nullptr;
    apply_observable(h, o, h->d_state, out, tmp);
    const double ms = norm2_of(h, out);
    double re, im;
    inner_of(h, h->d_state, out, &re, &im);
    return ms - re * re;
}

void check_handle(b200sv_state *h) { need(h != nullptr, "NULL state handle"); }

}  // namespace

int b200sv::run_guarded(const std::function<void()> &f) { return guard(f); }

// =============================================================================
extern "C" {

const char *b200sv_last_error(void) { return g_last_error.c_str(); }
int b200sv_version(void) { return 100; }

int b200sv_device_count(int *count) {
    return guard([&] {
        need(count != nullptr, "NULL output");
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess) {
            cudaGetLastError();
            n = 0;
        }
        *count = n;
    });
}

// The calls allocate their work buffers (lambda and bras of the adjoint, sampling and segment
// tables) stream-ordered from the device's default pool.  With the pool's default release
// threshold of 0, every synchronisation hands the freed memory back and the next call maps it
// again; keeping up to 1 GiB of freed memory in the pool (a setting of this process only) lets
// repeated calls reuse it.  A larger threshold set by the application is left as it is.
static void keep_pool_memory(int device) {
    static std::once_flag flags[64];
    if (device < 0 || device >= 64) return;
    std::call_once(flags[device], [device] {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        uint64_t cur = 0, want = uint64_t(1) << 30;
        if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &cur) == cudaSuccess && cur < want)
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &want);
        cudaGetLastError();
    });
}

int b200sv_create(uint32_t num_qubits, int dtype, b200sv_handle *out) {
    return guard([&] {
        need(out != nullptr, "NULL output handle");
        need(num_qubits >= 1 && num_qubits <= 36, "number of qubits must be in [1, 36]");
        need(dtype == B200SV_C64 || dtype == B200SV_C128, "dtype must be B200SV_C64 or B200SV_C128");
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
            cudaGetLastError();
            throw CudaError("no CUDA device is available (libb200sv has no CPU path)");
        }
        auto h = std::make_unique<b200sv_state>();
        h->nq = num_qubits;
        h->dtype = dtype;
        B200SV_CUDA(cudaGetDevice(&h->device));
        keep_pool_memory(h->device);
        try {
            B200SV_CUDA(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
            B200SV_CUDA(cudaMalloc(&h->d_state, h->state_bytes()));
            B200SV_CUDA(cudaMalloc(&h->d_partials, (kPartialsCapacity + 1) * sizeof(double)));
            B200SV_CUDA(cudaMemsetAsync(h->arrival(), 0, sizeof(double), h->own));
            B200SV_CUDA(cudaMalloc(&h->d_small, kSmall * sizeof(double)));
            B200SV_CUDA(cudaMallocHost(&h->h_small, kSmall * sizeof(double)));
            if (dtype == B200SV_C64) set_basis<float>(h->d_state, num_qubits, 0, h->own);
            else set_basis<double>(h->d_state, num_qubits, 0, h->own);
        } catch (...) {
            if (h->d_state) cudaFree(h->d_state);
            if (h->d_partials) cudaFree(h->d_partials);
            if (h->d_small) cudaFree(h->d_small);
            if (h->h_small) cudaFreeHost(h->h_small);
            if (h->own) cudaStreamDestroy(h->own);
            throw;
        }
        *out = h.release();
    });
}

int b200sv_destroy(b200sv_handle h) {
    return guard([&] {
        if (!h) return;
        DeviceGuard dg(h->device);
        cudaStreamSynchronize(h->stream());
        cudaFree(h->d_state);
        cudaFree(h->d_partials);
        cudaFree(h->d_small);
        cudaFreeHost(h->h_small);
        if (h->d_matrix) cudaFree(h->d_matrix);
        for (auto &s : h->d_scratch)
            if (s) cudaFree(s);
        for (int k = 0; k < 2; ++k) {
            if (h->h_stage[k]) cudaFreeHost(h->h_stage[k]);
            if (h->stage_ev[k]) cudaEventDestroy(h->stage_ev[k]);
        }
        cudaStreamDestroy(h->own);
        delete h;
    });
}

int b200sv_num_qubits(b200sv_handle h, uint32_t *out) {
    return guard([&] {
        check_handle(h);
        need(out != nullptr, "NULL output");
        *out = h->nq;
    });
}
int b200sv_dtype(b200sv_handle h, int *out) {
    return guard([&] {
        check_handle(h);
        need(out != nullptr, "NULL output");
        *out = h->dtype;
    });
}
int b200sv_set_stream(b200sv_handle h, void *s) {
    return guard([&] {
        check_handle(h);
        DeviceGuard dg(h->device);
        // on a change of stream, work issued on the previous one (the handle's initialisation
        // among it) completes before anything issued on the new one
        if (!h->has_ext || h->ext != static_cast<cudaStream_t>(s)) B200SV_CUDA(cudaStreamSynchronize(h->stream()));
        h->ext = static_cast<cudaStream_t>(s);
        h->has_ext = true;
    });
}
int b200sv_synchronize(b200sv_handle h) {
    return guard([&] {
        check_handle(h);
        DeviceGuard dg(h->device);
        B200SV_CUDA(cudaStreamSynchronize(h->stream()));
        if (dense_tc_timeouts() != 0)
            throw CudaError("a tensor-core matrix launch gave up waiting for its MMAs (results are invalid)");
    });
}
int b200sv_device_ptr(b200sv_handle h, void **out) {
    return guard([&] {
        check_handle(h);
        need(out != nullptr, "NULL output");
        *out = h->d_state;
    });
}
int b200sv_upload(b200sv_handle h, const void *host, uint64_t length) {
    return guard([&] {
        check_handle(h);
        need(host != nullptr, "NULL host buffer");
        need(length == (uint64_t(1) << h->nq), "length must equal 2^num_qubits");
        DeviceGuard dg(h->device);
        B200SV_CUDA(cudaMemcpyAsync(h->d_state, host, h->state_bytes(), cudaMemcpyHostToDevice, h->stream()));
        B200SV_CUDA(cudaStreamSynchronize(h->stream()));
    });
}
int b200sv_download(b200sv_handle h, void *host, uint64_t length) {
    return guard([&] {
        check_handle(h);
        need(host != nullptr, "NULL host buffer");
        need(length == (uint64_t(1) << h->nq), "length must equal 2^num_qubits");
        DeviceGuard dg(h->device);
        B200SV_CUDA(cudaMemcpyAsync(host, h->d_state, h->state_bytes(), cudaMemcpyDeviceToHost, h->stream()));
        B200SV_CUDA(cudaStreamSynchronize(h->stream()));
    });
}
int b200sv_copy(b200sv_handle dst, b200sv_handle src) {
    return guard([&] {
        check_handle(dst);
        check_handle(src);
        need(dst->nq == src->nq && dst->dtype == src->dtype, "copy needs equal size and dtype");
        DeviceGuard dg(dst->device);
        if (src->stream() != dst->stream()) B200SV_CUDA(cudaStreamSynchronize(src->stream()));
        B200SV_CUDA(cudaMemcpyAsync(dst->d_state, src->d_state, dst->state_bytes(), cudaMemcpyDeviceToDevice,
                                    dst->stream()));
    });
}
int b200sv_set_basis_state(b200sv_handle h, uint64_t index) {
    return guard([&] {
        check_handle(h);
        need(index < (uint64_t(1) << h->nq), "basis index out of range");
        DeviceGuard dg(h->device);
        if (h->dtype == B200SV_C64) set_basis<float>(h->d_state, h->nq, index, h->stream());
        else set_basis<double>(h->d_state, h->nq, index, h->stream());
    });
}

int b200sv_apply_gate(b200sv_handle h, uint32_t gate, const uint32_t *wires, uint32_t nwires, int inverse,
                      const double *params, uint32_t nparams) {
    return guard([&] {
        check_handle(h);
        need(nwires == 0 || wires, "NULL wires");
        need(nparams == 0 || params, "NULL params");
        DeviceGuard dg(h->device);
        GateDesc g = compile_gate(gate, wires, nwires, inverse != 0, params, nparams, h->nq);
        void *s[1] = {h->d_state};
        apply_desc(h, s, 1, g);
    });
}

int b200sv_apply_matrix(b200sv_handle h, const void *matrix, const uint32_t *wires, uint32_t nwires, int inverse) {
    return guard([&] {
        check_handle(h);
        need(matrix != nullptr && wires != nullptr, "NULL matrix or wires");
        need(nwires >= 1 && nwires <= 11, "applyMatrix supports 1..11 wires");
        DeviceGuard dg(h->device);
        const size_t d = size_t(1) << nwires;
        auto m = read_matrix(matrix, d * d, h->dtype);
        GateDesc g = compile_matrix(m.data(), wires, nwires, inverse != 0, h->nq);
        void *s[1] = {h->d_state};
        apply_desc(h, s, 1, g);
    });
}

int b200sv_apply_ops(b200sv_handle h, const b200sv_op *ops, uint32_t nops) {
    return guard([&] {
        check_handle(h);
        DeviceGuard dg(h->device);
        auto rec = read_ops(ops, nops, h->dtype);
        std::vector<GateDesc> descs;
        descs.reserve(rec.size());
        for (auto &o : rec) descs.push_back(compile_op(o, o.inverse, h->nq));  // validate all first
        void *s[1] = {h->d_state};
        for (auto &g : descs) apply_desc(h, s, 1, g);
    });
}

int b200sv_apply_ops_fused(b200sv_handle h, const b200sv_op *ops, uint32_t nops) {
    return guard([&] {
        check_handle(h);
        DeviceGuard dg(h->device);
        auto rec = read_ops(ops, nops, h->dtype);
        std::vector<GateDesc> descs;
        descs.reserve(rec.size());
        for (auto &o : rec) descs.push_back(compile_op(o, o.inverse, h->nq));  // validate all first
        void *s[1] = {h->d_state};
        if (!fused_worthwhile(h->dtype, h->nq)) {
            // too few tiles to fill the GPU: one launch per gate
            for (auto &g : descs) apply_desc(h, s, 1, g);
            return;
        }
        apply_fused(h->d_state, h->nq, h->dtype, descs, [&](const GateDesc &g) { apply_desc(h, s, 1, g); },
                    h->stream());
    });
}

int b200sv_apply_generator(b200sv_handle h, uint32_t generator, const uint32_t *wires, uint32_t nwires, int adj,
                           double *scale) {
    (void)adj;  // generators are Hermitian: adj does not change them (GateImplementationsLM.hpp:1355-1639)
    return guard([&] {
        check_handle(h);
        need(wires != nullptr && scale != nullptr, "NULL wires or scale");
        DeviceGuard dg(h->device);
        GateDesc g = compile_generator(generator, wires, nwires, h->nq, scale);
        void *s[1] = {h->d_state};
        apply_desc(h, s, 1, g);
    });
}

int b200sv_probs_device(b200sv_handle h, const uint32_t *wires, uint32_t nwires, double *out_device) {
    return guard([&] {
        check_handle(h);
        need(out_device != nullptr, "NULL output");
        DeviceGuard dg(h->device);
        std::vector<uint32_t> bits;
        if (nwires == 0) {
            for (uint32_t w = 0; w < h->nq; ++w) bits.push_back(bitpos(w, h->nq));
        } else {
            need(wires != nullptr, "NULL wires");
            check_wires(wires, nwires, h->nq, "probs");
            // Output bit r belongs to wire wires[s[s[r]]], s = argsort(wires): the
            // reference sums over the sorted wires and then applies
            // transpose_state_tensor(probs, s) (MeasurementsLQubit.hpp:98-136,
            // CS/utils/Util.hpp:465-496), which is this order.
            std::vector<uint32_t> s(nwires);
            for (uint32_t j = 0; j < nwires; ++j) s[j] = j;
            std::stable_sort(s.begin(), s.end(), [&](uint32_t a, uint32_t b) { return wires[a] < wires[b]; });
            for (uint32_t r = 0; r < nwires; ++r) bits.push_back(bitpos(wires[s[s[r]]], h->nq));
        }
        if (h->dtype == B200SV_C64)
            reduce_probs<float>(h->d_state, h->nq, bits, h->d_partials, kPartialsCapacity, out_device, h->stream());
        else
            reduce_probs<double>(h->d_state, h->nq, bits, h->d_partials, kPartialsCapacity, out_device, h->stream());
    });
}

int b200sv_probs(b200sv_handle h, const uint32_t *wires, uint32_t nwires, double *out) {
    return guard([&] {
        check_handle(h);
        need(out != nullptr, "NULL output");
        DeviceGuard dg(h->device);
        const uint32_t k = nwires == 0 ? h->nq : nwires;
        const size_t count = size_t(1) << k;
        double *d_out = nullptr;
        B200SV_CUDA(cudaMallocAsync((void **)&d_out, count * sizeof(double), h->stream()));
        int rc = b200sv_probs_device(h, wires, nwires, d_out);
        if (rc != B200SV_OK) {
            std::string msg = g_last_error;
            cudaFreeAsync(d_out, h->stream());
            throw ArgError(msg);
        }
        B200SV_CUDA(cudaMemcpyAsync(out, d_out, count * sizeof(double), cudaMemcpyDeviceToHost, h->stream()));
        B200SV_CUDA(cudaFreeAsync(d_out, h->stream()));
        B200SV_CUDA(cudaStreamSynchronize(h->stream()));
    });
}

int b200sv_apply_observable(b200sv_handle h, const b200sv_observable *obs) {
    return guard([&] {
        check_handle(h);
        need(obs != nullptr, "NULL observable");
        DeviceGuard dg(h->device);
        const ObsRec o = read_obs(*obs, h->nq, h->dtype);
        void *out = scratch(h, 0);
        void *tmp = o.terms.size() > 1 ? scratch(h, 1) : nullptr;
        apply_observable(h, o, h->d_state, out, tmp);
        B200SV_CUDA(cudaMemcpyAsync(h->d_state, out, h->state_bytes(), cudaMemcpyDeviceToDevice, h->stream()));
    });
}

int b200sv_expval(b200sv_handle h, const b200sv_observable *obs, double *out) {
    return guard([&] {
        check_handle(h);
        need(obs != nullptr && out != nullptr, "NULL observable or output");
        DeviceGuard dg(h->device);
        *out = expval_impl(h, read_obs(*obs, h->nq, h->dtype));
    });
}

int b200sv_var(b200sv_handle h, const b200sv_observable *obs, double *out) {
    return guard([&] {
        check_handle(h);
        need(obs != nullptr && out != nullptr, "NULL observable or output");
        DeviceGuard dg(h->device);
        *out = var_impl(h, read_obs(*obs, h->nq, h->dtype));
    });
}

int b200sv_expval_pauli(b200sv_handle h, uint32_t nterms, const double *coeffs, const uint32_t *offsets,
                        const uint32_t *wires, const char *paulis, double *out_terms, double *out_sum) {
    return guard([&] {
        check_handle(h);
        need(nterms == 0 || (offsets && coeffs), "NULL term arrays");
        DeviceGuard dg(h->device);
        std::vector<PauliWord> words(nterms);
        for (uint32_t t = 0; t < nterms; ++t) {
            need(offsets[t] <= offsets[t + 1], "Pauli offsets must be non-decreasing");
            uint64_t used = 0;
            for (uint32_t q = offsets[t]; q < offsets[t + 1]; ++q) {
                need(wires && paulis, "NULL wires or paulis");
                need(wires[q] < h->nq, "Pauli wire out of range");
                const uint64_t bit = uint64_t(1) << bitpos(wires[q], h->nq);
                need(!(used & bit), "All wires in observables must be disjoint.");
                used |= bit;
                switch (paulis[q]) {
                case 'I': break;
                case 'X': words[t].xmask |= bit; break;
                case 'Y': words[t].xmask |= bit; words[t].zmask |= bit; words[t].ny++; break;
                case 'Z': words[t].zmask |= bit; break;
                default: throw ArgError("Pauli letters must be I, X, Y or Z");
                }
            }
        }
        auto v = pauli_term_values(h, h->d_state, words);
        double s = 0.0;
        for (uint32_t t = 0; t < nterms; ++t) {
            if (out_terms) out_terms[t] = v[t];
            s += coeffs[t] * v[t];
        }
        if (out_sum) *out_sum = s;
    });
}

int b200sv_inner_product(b200sv_handle bra, b200sv_handle ket, double *re, double *im) {
    return guard([&] {
        check_handle(bra);
        check_handle(ket);
        need(re && im, "NULL output");
        need(bra->nq == ket->nq && bra->dtype == ket->dtype, "inner product needs equal size and dtype");
        DeviceGuard dg(ket->device);
        if (bra->stream() != ket->stream()) B200SV_CUDA(cudaStreamSynchronize(bra->stream()));
        inner_of(ket, bra->d_state, ket->d_state, re, im);
    });
}

int b200sv_norm2(b200sv_handle h, double *out) {
    return guard([&] {
        check_handle(h);
        need(out != nullptr, "NULL output");
        DeviceGuard dg(h->device);
        *out = norm2_of(h, h->d_state);
    });
}

// ---- host-array uploads ----------------------------------------------------------------
constexpr size_t kStageBytes = size_t(64) << 20;

// memcpy split over nt host threads
static void parallel_copy(char *dst, const char *src, size_t n, unsigned nt) {
    if (nt <= 1 || n < (size_t(1) << 20)) {
        std::memcpy(dst, src, n);
        return;
    }
    const size_t per = (n + nt - 1) / nt;
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t) {
        const size_t a = t * per;
        if (a >= n) break;
        const size_t b = std::min(n, a + per);
        th.emplace_back([=] { std::memcpy(dst + a, src + a, b - a); });
    }
    std::memcpy(dst, src, std::min(n, per));
    for (auto &x : th) x.join();
}

// Copy `bytes` from caller host memory to device memory on the state's stream.  Pinned (or
// registered) host memory is copied directly.  Large pageable arrays go through two pinned
// 64 MiB halves kept by the handle: host threads fill one half while the other half's copy
// runs, so the transfer runs near the pinned link rate instead of the pageable path's.  A half
// is refilled only after its previous copy has completed (an event per half), so the call may
// return while the last copies are still in flight.
static void upload_host(b200sv_state *h, void *dst, const void *src, size_t bytes) {
    if (!bytes) return;
    const cudaStream_t st = h->stream();
    cudaPointerAttributes pa{};
    const bool pinned = cudaPointerGetAttributes(&pa, src) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();  // a failed query of plain host memory leaves no error behind
    if (pinned || bytes <= (size_t(4) << 20)) {
        B200SV_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
        return;
    }
    for (int k = 0; k < 2; ++k) {
        if (!h->h_stage[k]) {
            if (cudaHostAlloc(&h->h_stage[k], kStageBytes, cudaHostAllocDefault) != cudaSuccess) {
                cudaGetLastError();
                h->h_stage[k] = nullptr;
                B200SV_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));  // no pinned memory
                return;
            }
        }
        if (!h->stage_ev[k]) B200SV_CUDA(cudaEventCreateWithFlags(&h->stage_ev[k], cudaEventDisableTiming));
    }
    const unsigned nt = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    const char *s = static_cast<const char *>(src);
    char *d = static_cast<char *>(dst);
    int k = 0;
    for (size_t off = 0; off < bytes; off += kStageBytes, k ^= 1) {
        const size_t n = std::min(kStageBytes, bytes - off);
        B200SV_CUDA(cudaEventSynchronize(h->stage_ev[k]));  // the half's previous copy has completed
        parallel_copy(static_cast<char *>(h->h_stage[k]), s + off, n, nt);
        B200SV_CUDA(cudaMemcpyAsync(d + off, h->h_stage[k], n, cudaMemcpyHostToDevice, st));
        B200SV_CUDA(cudaEventRecord(h->stage_ev[k], st));
    }
}

// ---- sparse Hamiltonian: LQ/measurements/MeasurementsLQubit.hpp:197-214, :451-472 ----
// out[0] = Re<psi|H psi>, out[1] = <H psi|H psi>.  The CSR arrays are checked on the host
// (the reference reads them unchecked) so no launch reads outside them or the state.
static void sparse_device(b200sv_state *h, const uint64_t *d_rows, const uint64_t *d_cols, const void *d_vals,
                          uint64_t nnz, double out[2]);

static void sparse_impl(b200sv_state *h, const uint64_t *row_map, uint64_t row_map_size, const uint64_t *entries,
                        const void *values, uint64_t nnz, double out[2]) {
    const uint64_t N = uint64_t(1) << h->nq;
    need(row_map != nullptr || row_map_size == 0, "NULL row_map");
    need(row_map_size >= 1 && row_map_size - 1 == N, "Statevector and Hamiltonian have incompatible sizes.");
    const uint64_t base = row_map[0];
    need(row_map[N] >= base, "row_map must be non-decreasing");
    const uint64_t used = row_map[N] - base;
    need(used <= nnz, "row_map addresses more non-zeros than the value array holds");
    need(used == 0 || (entries != nullptr && values != nullptr), "NULL entries or values");
    // the per-row bounds and column indices are checked on the device as the kernel reads them
    const cudaStream_t st = h->stream();
    const size_t S = h->dtype == B200SV_C64 ? 8 : 16;
    uint64_t *d_rows = nullptr, *d_cols = nullptr;
    void *d_vals = nullptr;
    B200SV_CUDA(cudaMallocAsync((void **)&d_rows, (N + 1) * sizeof(uint64_t), st));
    B200SV_CUDA(cudaMallocAsync((void **)&d_cols, std::max<uint64_t>(1, used) * sizeof(uint64_t), st));
    B200SV_CUDA(cudaMallocAsync(&d_vals, std::max<uint64_t>(1, used) * S, st));
    struct Free {
        void *a, *b, *c;
        cudaStream_t s;
        ~Free() {
            cudaFreeAsync(a, s);
            cudaFreeAsync(b, s);
            cudaFreeAsync(c, s);
        }
    } fr{d_rows, d_cols, d_vals, st};
    upload_host(h, d_rows, row_map, (N + 1) * sizeof(uint64_t));
    if (used) {
        upload_host(h, d_cols, entries, used * sizeof(uint64_t));
        upload_host(h, d_vals, values, used * S);
    }
    sparse_device(h, d_rows, d_cols, d_vals, used, out);
}

// CSR arrays in device memory: the kernel checks every row's bounds against [row_map[0],
// row_map[0] + nnz] and every column index, so nothing is read from the host.
static void sparse_device(b200sv_state *h, const uint64_t *d_rows, const uint64_t *d_cols, const void *d_vals,
                          uint64_t nnz, double out[2]) {
    const cudaStream_t st = h->stream();
    unsigned int *bad = reinterpret_cast<unsigned int *>(h->d_small + 2);
    B200SV_CUDA(cudaMemsetAsync(bad, 0, sizeof(double), st));
    if (h->dtype == B200SV_C64)
        reduce_sparse<float>(h->d_state, h->nq, d_rows, d_cols, d_vals, nnz, h->d_partials, h->d_small, bad, st);
    else
        reduce_sparse<double>(h->d_state, h->nq, d_rows, d_cols, d_vals, nnz, h->d_partials, h->d_small, bad, st);
    read_small(h, 2);
    unsigned int flags = 0;
    std::memcpy(&flags, &h->h_small[2], sizeof(flags));
    need(!(flags & 1u), "row_map must be non-decreasing");
    need(!(flags & 4u), "row_map addresses more non-zeros than the value array holds");
    need(!(flags & 2u), "sparse column index out of range");
    out[0] = h->h_small[0];
    out[1] = h->h_small[1];
}

int b200sv_expval_sparse_device(b200sv_handle h, const uint64_t *row_map, const uint64_t *entries,
                                const void *values, uint64_t nnz, double *out) {
    return guard([&] {
        check_handle(h);
        need(out != nullptr && row_map != nullptr, "NULL row_map or output");
        need(nnz == 0 || (entries != nullptr && values != nullptr), "NULL entries or values");
        DeviceGuard dg(h->device);
        double r[2];
        sparse_device(h, row_map, entries, values, nnz, r);
        *out = r[0];
    });
}

int b200sv_var_sparse_device(b200sv_handle h, const uint64_t *row_map, const uint64_t *entries,
                             const void *values, uint64_t nnz, double *out) {
    return guard([&] {
        check_handle(h);
        need(out != nullptr && row_map != nullptr, "NULL row_map or output");
        need(nnz == 0 || (entries != nullptr && values != nullptr), "NULL entries or values");
        DeviceGuard dg(h->device);
        double r[2];
        sparse_device(h, row_map, entries, values, nnz, r);
        *out = r[1] - r[0] * r[0];
    });
}

int b200sv_expval_sparse(b200sv_handle h, const uint64_t *row_map, uint64_t row_map_size, const uint64_t *entries,
                         const void *values, uint64_t nnz, double *out) {
    return guard([&] {
        check_handle(h);
        need(out != nullptr, "NULL output");
        DeviceGuard dg(h->device);
        double r[2];
        sparse_impl(h, row_map, row_map_size, entries, values, nnz, r);
        *out = r[0];
    });
}

int b200sv_var_sparse(b200sv_handle h, const uint64_t *row_map, uint64_t row_map_size, const uint64_t *entries,
                      const void *values, uint64_t nnz, double *out) {
    return guard([&] {
        check_handle(h);
        need(out != nullptr, "NULL output");
        DeviceGuard dg(h->device);
        double r[2];
        sparse_impl(h, row_map, row_map_size, entries, values, nnz, r);
        *out = r[1] - r[0] * r[0];
    });
}

static void sample_impl(b200sv_state *h, uint64_t nshots, const double *uniforms, uint64_t seed, uint64_t *idx_host) {
    const cudaStream_t st = h->stream();
    const uint64_t N = uint64_t(1) << h->nq;
    const size_t ws = run_offsets_doubles(N);
    double *work = nullptr, *u = nullptr;
    uint64_t *idx = nullptr;
    B200SV_CUDA(cudaMallocAsync((void **)&work, ws * sizeof(double), st));
    B200SV_CUDA(cudaMallocAsync((void **)&u, std::max<uint64_t>(1, nshots) * sizeof(double), st));
    B200SV_CUDA(cudaMallocAsync((void **)&idx, std::max<uint64_t>(1, nshots) * sizeof(uint64_t), st));
    if (h->dtype == B200SV_C64) build_run_offsets<float>(h->d_state, h->nq, work, st);
    else build_run_offsets<double>(h->d_state, h->nq, work, st);
    if (uniforms) B200SV_CUDA(cudaMemcpyAsync(u, uniforms, nshots * sizeof(double), cudaMemcpyHostToDevice, st));
    else philox_uniforms(u, nshots, seed, st);
    if (h->dtype == B200SV_C64) sample_runs<float>(h->d_state, h->nq, work, u, nshots, idx, st);
    else sample_runs<double>(h->d_state, h->nq, work, u, nshots, idx, st);
    if (nshots) B200SV_CUDA(cudaMemcpyAsync(idx_host, idx, nshots * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    cudaFreeAsync(work, st);
    cudaFreeAsync(u, st);
    cudaFreeAsync(idx, st);
    B200SV_CUDA(cudaStreamSynchronize(st));
}

int b200sv_sample(b200sv_handle h, uint64_t nshots, const double *uniforms, uint64_t seed, uint64_t *idx_out) {
    return guard([&] {
        check_handle(h);
        need(nshots == 0 || idx_out != nullptr, "NULL output");
        DeviceGuard dg(h->device);
        sample_impl(h, nshots, uniforms, seed, idx_out);
    });
}

int b200sv_sample_bits(b200sv_handle h, uint64_t nshots, const double *uniforms, uint64_t seed, uint64_t *bits_out) {
    return guard([&] {
        check_handle(h);
        need(nshots == 0 || bits_out != nullptr, "NULL output");
        DeviceGuard dg(h->device);
        std::vector<uint64_t> idx(nshots);
        sample_impl(h, nshots, uniforms, seed, idx.data());
        const uint32_t n = h->nq;
        // bits MSB (wire 0) first, as MeasurementsLQubit.hpp:549-554
        for (uint64_t s = 0; s < nshots; ++s)
            for (uint32_t j = 0; j < n; ++j) bits_out[s * n + (n - 1 - j)] = (idx[s] >> j) & 1u;
    });
}

int b200sv_sample_mcmc(b200sv_handle h, int proposal, uint64_t num_burnin, uint64_t nshots, uint32_t nchains,
                       uint64_t seed, uint64_t *idx_out) {
    return guard([&] {
        check_handle(h);
        need(nshots == 0 || idx_out != nullptr, "NULL output");
        DeviceGuard dg(h->device);
        const cudaStream_t st = h->stream();
        uint64_t *idx = nullptr;
        B200SV_CUDA(cudaMallocAsync((void **)&idx, std::max<uint64_t>(1, nshots) * sizeof(uint64_t), st));
        struct Free {
            uint64_t *p;
            cudaStream_t s;
            ~Free() { cudaFreeAsync(p, s); }
        } fr{idx, st};
        sample_mcmc(h->d_state, h->nq, h->dtype, proposal, num_burnin, nshots, nchains, seed, idx, st);
        if (nshots) B200SV_CUDA(cudaMemcpyAsync(idx_out, idx, nshots * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
        B200SV_CUDA(cudaStreamSynchronize(st));
    });
}

// The 2x2 matrix of a one-wire descriptor without controls; false for other forms.
static bool as_one_wire(const GateDesc &g, cd (&m)[4]) {
    if (g.tbits.size() != 1 || !g.cbits.empty() || g.k != 1) return false;
    switch (g.kind) {
    case Kind::Dense:
        for (int i = 0; i < 4; ++i) m[i] = g.m[i];
        return true;
    case Kind::Diag:
        m[0] = g.m[0];
        m[1] = m[2] = cd(0.0, 0.0);
        m[3] = g.m[1];
        return true;
    case Kind::Swap:
        m[0] = m[3] = cd(0.0, 0.0);
        m[1] = m[2] = cd(1.0, 0.0);
        return g.sa != g.sb;
    default: return false;
    }
}

// ---- adjoint Jacobian: LQ/algorithms/AdjointJacobianLQubit.hpp:212-335 --------
int b200sv_adjoint_jacobian(b200sv_handle psi, const b200sv_op *ops, uint32_t nops, const b200sv_observable *obs,
                            uint32_t nobs, const uint64_t *trainable, uint32_t ntp, int apply_operations,
                            double *jac) {
    return guard([&] {
        check_handle(psi);
        need(nobs == 0 || obs != nullptr, "NULL observables");
        need(ntp == 0 || trainable != nullptr, "NULL trainable parameter list");
        need(ntp == 0 || nobs == 0 || jac != nullptr, "NULL jacobian output");
        if (ntp == 0) return;  // nothing to do (AdjointJacobianLQubit.hpp:229-231)
        for (uint32_t i = 1; i < ntp; ++i) need(trainable[i - 1] < trainable[i], "trainable parameters must be sorted");
        DeviceGuard dg(psi->device);
        b200sv_state *h = psi;
        const cudaStream_t st = h->stream();
        auto rec = read_ops(ops, nops, h->dtype);
        std::vector<ObsRec> orec;
        for (uint32_t o = 0; o < nobs; ++o) orec.push_back(read_obs(obs[o], h->nq, h->dtype));
        size_t num_param_ops = 0;
        for (auto &o : rec)
            if (!o.params.empty()) ++num_param_ops;

        // workspace: lambda, one bra per observable, a tmp, the jacobian [tp][obs]
        std::vector<void *> bufs;
        auto alloc_state = [&]() {
            void *p = nullptr;
            B200SV_CUDA(cudaMallocAsync(&p, h->state_bytes(), st));
            bufs.push_back(p);
            return p;
        };
        double *d_jac = nullptr;
        struct Cleanup {
            std::vector<void *> &b;
            double *&j;
            cudaStream_t s;
            ~Cleanup() {
                for (auto p : b) cudaFreeAsync(p, s);
                if (j) cudaFreeAsync(j, s);
                cudaStreamSynchronize(s);
            }
        } cleanup{bufs, d_jac, st};
        void *lambda = alloc_state();
        std::vector<void *> bras;
        for (uint32_t o = 0; o < nobs; ++o) bras.push_back(alloc_state());
        bool need_tmp = false;
        for (auto &o : orec) need_tmp |= o.terms.size() > 1;
        void *tmp = need_tmp ? alloc_state() : nullptr;
        B200SV_CUDA(cudaMallocAsync((void **)&d_jac, sizeof(double) * ntp * std::max<uint32_t>(1, nobs), st));
        B200SV_CUDA(cudaMemsetAsync(d_jac, 0, sizeof(double) * ntp * std::max<uint32_t>(1, nobs), st));

        B200SV_CUDA(cudaMemcpyAsync(lambda, h->d_state, h->state_bytes(), cudaMemcpyDeviceToDevice, st));
        if (apply_operations) {
            std::vector<GateDesc> fwd;
            for (auto &o : rec) fwd.push_back(compile_op(o, o.inverse, h->nq));
            void *s1[1] = {lambda};
            if (fused_worthwhile(h->dtype, h->nq))
                apply_fused(lambda, h->nq, h->dtype, fwd, [&](const GateDesc &g) { apply_desc(h, s1, 1, g); }, st);
            else
                for (auto &g : fwd) apply_desc(h, s1, 1, g);
        }
        for (uint32_t o = 0; o < nobs; ++o) apply_observable(h, orec[o], lambda, bras[o], tmp);

        // the reverse sweep as a list of steps, with the reference's bookkeeping: reverse
        // traversal, trainable-parameter cursor, early exit once every trainable parameter is done
        std::vector<AdjItem> items;
        {
            int64_t tp_pos = (int64_t)ntp - 1;  // reverse iterator over trainable
            int64_t trainable_number = (int64_t)ntp - 1;
            int64_t current_param_idx = (int64_t)num_param_ops - 1;
            for (int64_t op_idx = (int64_t)rec.size() - 1; op_idx >= 0; --op_idx) {
                const OpRec &op = rec[op_idx];
                if (op.params.size() > 1)
                    throw ArgError("The operation is not supported using the adjoint differentiation method");
                if (op.gate == B200SV_OP_SKIP) continue;
                if (tp_pos < 0) break;
                AdjItem it;
                it.adj = compile_op(op, !op.inverse, h->nq);
                if (!op.params.empty()) {
                    if ((uint64_t)current_param_idx == trainable[tp_pos]) {
                        const int gen = generator_of_gate(op.gate);
                        if (gen < 0)
                            throw ArgError("The operation is not supported using the adjoint differentiation method");
                        double sc = 0.0;
                        it.G = compile_generator((uint32_t)gen, op.wires.data(), (uint32_t)op.wires.size(), h->nq, &sc);
                        it.diff = true;
                        it.alpha = -2.0 * sc * (op.inverse ? -1.0 : 1.0);
                        it.col = trainable_number;
                        --trainable_number;
                        --tp_pos;
                    }
                    --current_param_idx;
                }
                items.push_back(std::move(it));
            }
        }
        std::vector<void *> lambda_and_bras{lambda};
        lambda_and_bras.insert(lambda_and_bras.end(), bras.begin(), bras.end());
        // one step: the products (one-wire gates: products and inverse in one pass over the pairs)
        auto exec_single = [&](size_t i) {
            const AdjItem &it = items[i];
            if (it.diff) {
                cd g2[4], u2[4];
                if (nobs >= 1 && nobs <= 16 && as_one_wire(it.G, g2) && as_one_wire(it.adj, u2) &&
                    it.G.tbits[0] == it.adj.tbits[0]) {
                    double *dst = d_jac + (size_t)it.col * nobs;
                    if (h->dtype == B200SV_C64)
                        adjoint_rot_step<float>(lambda, bras.data(), (int)nobs, h->nq, it.G.tbits[0], g2, u2, it.alpha,
                                                h->d_partials, dst, 1, h->arrival(), st);
                    else
                        adjoint_rot_step<double>(lambda, bras.data(), (int)nobs, h->nq, it.G.tbits[0], g2, u2, it.alpha,
                                                 h->d_partials, dst, 1, h->arrival(), st);
                    return;
                }
                for (uint32_t o0 = 0; o0 < nobs; o0 += 16) {
                    const int cnt = (int)std::min<uint32_t>(16, nobs - o0);
                    double *dst = d_jac + (size_t)it.col * nobs + o0;
                    if (h->dtype == B200SV_C64)
                        reduce_generator_inner<float>(bras.data() + o0, cnt, lambda, h->nq, it.G, it.alpha,
                                                      h->d_partials, dst, 1, st, h->arrival());
                    else
                        reduce_generator_inner<double>(bras.data() + o0, cnt, lambda, h->nq, it.G, it.alpha,
                                                       h->d_partials, dst, 1, st, h->arrival());
                }
            }
            apply_desc_multi(h, lambda_and_bras, it.adj);  // lambda and every bra in one launch
        };
        if (nobs == 1 && fused_adjoint_worthwhile(h->dtype, h->nq)) {
            // one bra (the VJP form): fused passes over lambda and the bra
            apply_fused_adjoint(lambda, bras[0], h->nq, h->dtype, items, exec_single, d_jac, st);
        } else {
            for (size_t i = 0; i < items.size(); ++i) exec_single(i);
        }
        std::vector<double> jt((size_t)ntp * nobs);
        if (!jt.empty())
            B200SV_CUDA(cudaMemcpyAsync(jt.data(), d_jac, jt.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        B200SV_CUDA(cudaStreamSynchronize(st));
        // [tp][obs] -> [obs][tp]  (AdjointJacobianLQubit.hpp:331-334)
        for (uint32_t p = 0; p < ntp; ++p)
            for (uint32_t o = 0; o < nobs; ++o) jac[(size_t)o * ntp + p] = jt[(size_t)p * nobs + o];
    });
}

// ---- state-return VJP: LQ/algorithms/VectorJacobianProduct.hpp:60-156 --------
int b200sv_vjp_state(b200sv_handle psi, const b200sv_op *ops, uint32_t nops, const void *dy, uint64_t dy_length,
                     const uint64_t *trainable, uint32_t ntp, int apply_operations, double *out) {
    return guard([&] {
        check_handle(psi);
        need(dy != nullptr, "NULL cotangent state");
        need(dy_length == (uint64_t(1) << psi->nq), "dy must have 2^num_qubits entries");
        need(ntp == 0 || (trainable && out), "NULL trainable list or output");
        if (ntp == 0) return;
        for (uint32_t i = 1; i < ntp; ++i) need(trainable[i - 1] < trainable[i], "trainable parameters must be sorted");
        DeviceGuard dg(psi->device);
        b200sv_state *h = psi;
        const cudaStream_t st = h->stream();
        auto rec = read_ops(ops, nops, h->dtype);
        size_t num_param_ops = 0;
        for (auto &o : rec)
            if (!o.params.empty()) ++num_param_ops;
        void *lambda = nullptr, *mu = nullptr;
        double *d_z = nullptr;
        B200SV_CUDA(cudaMallocAsync(&lambda, h->state_bytes(), st));
        B200SV_CUDA(cudaMallocAsync(&mu, h->state_bytes(), st));
        B200SV_CUDA(cudaMallocAsync((void **)&d_z, sizeof(double) * 2 * ntp, st));
        struct Cleanup {
            void *a, *b;
            double *z;
            cudaStream_t s;
            ~Cleanup() {
                cudaFreeAsync(a, s);
                cudaFreeAsync(b, s);
                cudaFreeAsync(z, s);
                cudaStreamSynchronize(s);
            }
        } cleanup{lambda, mu, d_z, st};
        B200SV_CUDA(cudaMemsetAsync(d_z, 0, sizeof(double) * 2 * ntp, st));
        B200SV_CUDA(cudaMemcpyAsync(lambda, h->d_state, h->state_bytes(), cudaMemcpyDeviceToDevice, st));
        B200SV_CUDA(cudaMemcpyAsync(mu, dy, h->state_bytes(), cudaMemcpyHostToDevice, st));
        if (apply_operations) {
            for (auto &o : rec) {
                void *s1[1] = {lambda};
                apply_desc(h, s1, 1, compile_op(o, o.inverse, h->nq));
            }
        }
        std::vector<double> scale(ntp, 0.0);
        int64_t tp_pos = (int64_t)ntp - 1;
        int64_t current = (int64_t)num_param_ops - 1;
        for (int64_t op_idx = (int64_t)rec.size() - 1; op_idx >= 0; --op_idx) {
            const OpRec &op = rec[op_idx];
            if (op.params.size() > 1)
                throw ArgError("The operation is not supported using the adjoint differentiation method");
            if (op.gate == B200SV_OP_SKIP) continue;
            if (tp_pos < 0) break;
            if (!op.params.empty()) {
                if ((uint64_t)current == trainable[tp_pos]) {
                    const int gen = generator_of_gate(op.gate);
                    if (gen < 0)
                        throw ArgError("The operation is not supported using the adjoint differentiation method");
                    double sc = 0.0;
                    GateDesc G = compile_generator((uint32_t)gen, op.wires.data(), (uint32_t)op.wires.size(), h->nq, &sc);
                    scale[tp_pos] = sc * (op.inverse ? -1.0 : 1.0);
                    if (h->dtype == B200SV_C64)
                        reduce_generator_inner_complex<float>(mu, lambda, h->nq, G, h->d_partials, d_z + 2 * tp_pos, st);
                    else
                        reduce_generator_inner_complex<double>(mu, lambda, h->nq, G, h->d_partials, d_z + 2 * tp_pos, st);
                    --tp_pos;
                }
                --current;
            }
            GateDesc adj = compile_op(op, !op.inverse, h->nq);
            void *two[2] = {lambda, mu};
            apply_desc(h, two, 2, adj);
        }
        std::vector<double> z(2 * ntp);
        B200SV_CUDA(cudaMemcpyAsync(z.data(), d_z, z.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        B200SV_CUDA(cudaStreamSynchronize(st));
        for (uint32_t j = 0; j < ntp; ++j) {  // i * scale * z
            out[2 * j] = -scale[j] * z[2 * j + 1];
            out[2 * j + 1] = scale[j] * z[2 * j];
        }
    });
}

}  // extern "C"
