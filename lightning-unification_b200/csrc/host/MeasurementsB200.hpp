// MeasurementsB200.hpp — Measurements<StateVectorT> of lightning.qubit
// (LQ/measurements/MeasurementsLQubit.hpp:61-641, CS/measurements/MeasurementsBase.hpp:42-106)
// on the C ABI.  Expectation values are fused read-only reductions on the
// device instead of copy + apply + inner product.
#pragma once

#include <random>

#include "ObservablesB200.hpp"

namespace Pennylane::LightningB200 {

template <class StateVectorT> class Measurements {
    using PrecisionT = typename StateVectorT::PrecisionT;
    using ComplexT = typename StateVectorT::ComplexT;
    const StateVectorT &sv_;

    PrecisionT run_expval(const std::vector<TermData<PrecisionT>> &t) const {
        ObsRecord<PrecisionT> r(t);
        double out = 0;
        check(b200sv_expval(sv_.handle(), &r.rec, &out));
        return (PrecisionT)out;
    }
    PrecisionT run_var(const std::vector<TermData<PrecisionT>> &t) const {
        ObsRecord<PrecisionT> r(t);
        double out = 0;
        check(b200sv_var(sv_.handle(), &r.rec, &out));
        return (PrecisionT)out;
    }

    template <class index_type>
    double run_sparse(const index_type *rows, index_type nrows, const index_type *cols, const ComplexT *vals,
                      index_type nnz, bool variance) const {
        std::vector<uint64_t> r(rows, rows + nrows), c(cols, cols + std::min<index_type>(nnz, nrows ? rows[nrows - 1] - rows[0] : 0));
        double out = 0;
        check((variance ? b200sv_var_sparse : b200sv_expval_sparse)(sv_.handle(), r.data(), (uint64_t)nrows, c.data(),
                                                                     vals, (uint64_t)nnz, &out));
        return out;
    }

  public:
    explicit Measurements(const StateVectorT &sv) : sv_(sv) {}

    // :79-88
    std::vector<PrecisionT> probs() const { return probs({}); }
    // :98-136 (wires[0] is the most significant bit of the result index)
    std::vector<PrecisionT> probs(const std::vector<size_t> &wires) const {
        std::vector<uint32_t> w(wires.begin(), wires.end());
        const size_t k = wires.empty() ? sv_.getNumQubits() : wires.size();
        std::vector<double> out(size_t(1) << k);
        check(b200sv_probs(sv_.handle(), w.data(), (uint32_t)w.size(), out.data()));
        return {out.begin(), out.end()};
    }
    // :167-180
    PrecisionT expval(const std::string &name, const std::vector<size_t> &wires) const {
        return run_expval({TermData<PrecisionT>{1.0, {FactorData<PrecisionT>{true, name, wires, {}}}}});
    }
    // :145-158
    PrecisionT expval(const std::vector<ComplexT> &matrix, const std::vector<size_t> &wires) const {
        return run_expval({TermData<PrecisionT>{1.0, {FactorData<PrecisionT>{false, "Hermitian", wires, matrix}}}});
    }
    // :248-265
    PrecisionT expval(const Observable<StateVectorT> &ob) const { return run_expval(ob.terms()); }
    // :218-240
    template <typename op_type>
    std::vector<PrecisionT> expval(const std::vector<op_type> &ops, const std::vector<std::vector<size_t>> &wires) const {
        if (ops.size() != wires.size())
            throw LightningException("The lengths of the list of operations and wires do not match.");
        std::vector<PrecisionT> r;
        for (size_t i = 0; i < ops.size(); ++i) r.push_back(expval(ops[i], wires[i]));
        return r;
    }
    // :273-372
    PrecisionT var(const Observable<StateVectorT> &ob) const { return run_var(ob.terms()); }
    PrecisionT var(const std::string &name, const std::vector<size_t> &wires) const {
        return run_var({TermData<PrecisionT>{1.0, {FactorData<PrecisionT>{true, name, wires, {}}}}});
    }
    PrecisionT var(const std::vector<ComplexT> &matrix, const std::vector<size_t> &wires) const {
        return run_var({TermData<PrecisionT>{1.0, {FactorData<PrecisionT>{false, "Hermitian", wires, matrix}}}});
    }
    // :197-214 (CSR sparse Hamiltonian; values in the state's precision)
    template <class index_type>
    PrecisionT expval(const index_type *row_map_ptr, const index_type row_map_size, const index_type *entries_ptr,
                      const ComplexT *values_ptr, const index_type numNNZ) const {
        return (PrecisionT)run_sparse(row_map_ptr, row_map_size, entries_ptr, values_ptr, numNNZ, false);
    }
    // :451-472
    template <class index_type>
    PrecisionT var(const index_type *row_map_ptr, const index_type row_map_size, const index_type *entries_ptr,
                   const ComplexT *values_ptr, const index_type numNNZ) const {
        return (PrecisionT)run_sparse(row_map_ptr, row_map_size, entries_ptr, values_ptr, numNNZ, true);
    }
    // generate_samples (:482-558 signature and output layout; sampling rule of
    // LK/measurements/MeasuresFunctors.hpp:70-103 with device Philox draws).
    std::vector<size_t> generate_samples(size_t num_samples, uint64_t seed) const {
        const size_t n = sv_.getNumQubits();
        std::vector<uint64_t> bits(num_samples * n);
        check(b200sv_sample_bits(sv_.handle(), num_samples, nullptr, seed, bits.data()));
        return {bits.begin(), bits.end()};
    }
    std::vector<size_t> generate_samples(size_t num_samples) const {
        return generate_samples(num_samples, std::random_device{}());
    }
    // generate_samples_metropolis (:387-434): bits of num_samples indices, wire 0 first.
    // The kernel name is bound to a proposal as the reference binds it (kernel_factory,
    // TransitionKernels.hpp:147-159: "NonZeroRandom" runs the local proposal, any other
    // name the non-zero one).  num_chains independent chains share the samples.
    std::vector<size_t> generate_samples_metropolis(const std::string &kernelname, size_t num_burnin,
                                                    size_t num_samples, uint64_t seed,
                                                    uint32_t num_chains = 4096) const {
        const size_t n = sv_.getNumQubits();
        const int proposal = kernelname == "NonZeroRandom" ? B200SV_MCMC_LOCAL : B200SV_MCMC_NONZERO;
        std::vector<uint64_t> idx(num_samples);
        check(b200sv_sample_mcmc(sv_.handle(), proposal, num_burnin, num_samples, num_chains, seed, idx.data()));
        std::vector<size_t> bits(num_samples * n);
        for (size_t s = 0; s < num_samples; ++s)
            for (size_t j = 0; j < n; ++j) bits[s * n + (n - 1 - j)] = (idx[s] >> j) & 1u;
        return bits;
    }
    std::vector<size_t> generate_samples_metropolis(const std::string &kernelname, size_t num_burnin,
                                                    size_t num_samples) const {
        return generate_samples_metropolis(kernelname, num_burnin, num_samples, std::random_device{}());
    }
    // seeded variant taking caller uniforms (bit-exact reproducibility)
    std::vector<size_t> generate_samples_from_uniforms(const std::vector<double> &u) const {
        const size_t n = sv_.getNumQubits();
        std::vector<uint64_t> bits(u.size() * n);
        check(b200sv_sample_bits(sv_.handle(), u.size(), u.data(), 0, bits.data()));
        return {bits.begin(), bits.end()};
    }
};

}  // namespace Pennylane::LightningB200
