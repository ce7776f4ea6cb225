// AdjointJacobianB200.hpp — OpsData, JacobianData and AdjointJacobian of lightning.qubit
// (CS/algorithms/JacobianData.hpp:40-336, LQ/algorithms/AdjointJacobianLQubit.hpp:212-335)
// driving b200sv_adjoint_jacobian.
#pragma once

#include <numeric>

#include "ObservablesB200.hpp"

namespace Pennylane::LightningB200 {

template <class StateVectorT> class OpsData {
    using PrecisionT = typename StateVectorT::PrecisionT;
    using ComplexT = typename StateVectorT::ComplexT;
    size_t num_par_ops_ = 0;
    std::vector<std::string> name_;
    std::vector<std::vector<PrecisionT>> params_;
    std::vector<std::vector<size_t>> wires_;
    std::vector<bool> inv_;
    std::vector<std::vector<ComplexT>> mats_;

  public:
    OpsData(std::vector<std::string> names, std::vector<std::vector<PrecisionT>> params,
            std::vector<std::vector<size_t>> wires, std::vector<bool> inverses,
            std::vector<std::vector<ComplexT>> matrices = {})
        : name_(std::move(names)), params_(std::move(params)), wires_(std::move(wires)), inv_(std::move(inverses)),
          mats_(std::move(matrices)) {
        if (mats_.empty()) mats_.resize(name_.size());
        if (params_.size() != name_.size() || wires_.size() != name_.size() || inv_.size() != name_.size() ||
            mats_.size() != name_.size())
            throw LightningException("OpsData: all operation lists must have the same length");
        for (auto &p : params_) num_par_ops_ += p.empty() ? 0 : 1;
    }
    [[nodiscard]] size_t getSize() const { return name_.size(); }
    [[nodiscard]] const std::vector<std::string> &getOpsName() const { return name_; }
    [[nodiscard]] const std::vector<std::vector<PrecisionT>> &getOpsParams() const { return params_; }
    [[nodiscard]] const std::vector<std::vector<size_t>> &getOpsWires() const { return wires_; }
    [[nodiscard]] const std::vector<bool> &getOpsInverses() const { return inv_; }
    [[nodiscard]] const std::vector<std::vector<ComplexT>> &getOpsMatrices() const { return mats_; }
    [[nodiscard]] bool hasParams(size_t i) const { return !params_[i].empty(); }
    [[nodiscard]] size_t getNumParOps() const { return num_par_ops_; }
    [[nodiscard]] size_t getNumNonParOps() const { return name_.size() - num_par_ops_; }
    [[nodiscard]] size_t getTotalNumParams() const {
        size_t s = 0;
        for (auto &p : params_) s += p.size();
        return s;
    }
};

template <class StateVectorT> class JacobianData {
    using ComplexT = typename StateVectorT::ComplexT;
    size_t num_parameters_, num_elements_;
    const ComplexT *psi_;
    std::vector<std::shared_ptr<Observable<StateVectorT>>> obs_;
    OpsData<StateVectorT> ops_;
    std::vector<size_t> tp_;

  public:
    JacobianData(size_t num_params, size_t num_elem, const ComplexT *psi,
                 std::vector<std::shared_ptr<Observable<StateVectorT>>> obs, OpsData<StateVectorT> ops,
                 std::vector<size_t> trainP)
        : num_parameters_(num_params), num_elements_(num_elem), psi_(psi), obs_(std::move(obs)), ops_(std::move(ops)),
          tp_(std::move(trainP)) {}
    [[nodiscard]] size_t getNumParams() const { return num_parameters_; }
    [[nodiscard]] size_t getSizeStateVec() const { return num_elements_; }
    [[nodiscard]] const ComplexT *getPtrStateVec() const { return psi_; }
    [[nodiscard]] const std::vector<std::shared_ptr<Observable<StateVectorT>>> &getObservables() const { return obs_; }
    [[nodiscard]] size_t getNumObservables() const { return obs_.size(); }
    [[nodiscard]] const OpsData<StateVectorT> &getOperations() const { return ops_; }
    [[nodiscard]] const std::vector<size_t> &getTrainableParams() const { return tp_; }
    [[nodiscard]] bool hasTrainableParams() const { return !tp_.empty(); }
};

template <class StateVectorT> class AdjointJacobian {
    using PrecisionT = typename StateVectorT::PrecisionT;

  public:
    // jac: [observable][trainable parameter] (AdjointJacobianLQubit.hpp:331-334).
    // When jd's state pointer is null, `device_psi` supplies the state directly
    // on the device (no host round trip).
    void adjointJacobian(std::span<PrecisionT> jac, const JacobianData<StateVectorT> &jd,
                         bool apply_operations = false, const StateVectorT *device_psi = nullptr) {
        const auto &ops = jd.getOperations();
        const auto &tp = jd.getTrainableParams();
        const size_t nobs = jd.getNumObservables();
        if (!jd.hasTrainableParams()) return;
        if (jac.size() != tp.size() * nobs)
            throw LightningException("The size of preallocated jacobian must be same as the number of trainable "
                                     "parameters times the number of observables provided.");
        std::unique_ptr<StateVectorT> owned;
        const StateVectorT *sv = device_psi;
        if (!sv) {
            owned = std::make_unique<StateVectorT>(jd.getPtrStateVec(), jd.getSizeStateVec());
            sv = owned.get();
        }
        // operations
        std::vector<b200sv_op> cops(ops.getSize());
        std::vector<std::vector<uint32_t>> w(ops.getSize());
        std::vector<std::vector<double>> p(ops.getSize());
        for (size_t i = 0; i < ops.getSize(); ++i) {
            w[i].assign(ops.getOpsWires()[i].begin(), ops.getOpsWires()[i].end());
            p[i].assign(ops.getOpsParams()[i].begin(), ops.getOpsParams()[i].end());
            const bool has_mat = !ops.getOpsMatrices()[i].empty();
            cops[i].gate = has_mat ? (uint32_t)B200SV_OP_MATRIX : op_id(ops.getOpsName()[i]);
            cops[i].nwires = (uint32_t)w[i].size();
            cops[i].wires = w[i].data();
            cops[i].inverse = ops.getOpsInverses()[i] ? 1 : 0;
            cops[i].nparams = (uint32_t)p[i].size();
            cops[i].params = p[i].data();
            cops[i].matrix = has_mat ? ops.getOpsMatrices()[i].data() : nullptr;
        }
        // observables
        std::vector<std::unique_ptr<ObsRecord<PrecisionT>>> recs;
        std::vector<b200sv_observable> cobs;
        for (auto &o : jd.getObservables()) {
            recs.push_back(std::make_unique<ObsRecord<PrecisionT>>(o->terms()));
            cobs.push_back(recs.back()->rec);
        }
        std::vector<uint64_t> tpu(tp.begin(), tp.end());
        std::vector<double> out(jac.size());
        check(b200sv_adjoint_jacobian(sv->handle(), cops.data(), (uint32_t)cops.size(), cobs.data(),
                                      (uint32_t)cobs.size(), tpu.data(), (uint32_t)tpu.size(),
                                      apply_operations ? 1 : 0, out.data()));
        for (size_t i = 0; i < jac.size(); ++i) jac[i] = (PrecisionT)out[i];
    }
};

// VectorJacobianProduct (LQ/algorithms/VectorJacobianProduct.hpp:60-156): jac[j] = i * scale *
// <G mu | lambda> with mu the cotangent state dy, both swept backwards.
template <class StateVectorT> class VectorJacobianProduct {
    using PrecisionT = typename StateVectorT::PrecisionT;
    using ComplexT = typename StateVectorT::ComplexT;

  public:
    void operator()(std::span<ComplexT> jac, const JacobianData<StateVectorT> &jd, std::span<const ComplexT> dy,
                    bool apply_operations = false, const StateVectorT *device_psi = nullptr) {
        if (dy.size() != jd.getSizeStateVec()) throw LightningException("Assertion failed: dy.size() == jd.getSizeStateVec()");
        const auto &tp = jd.getTrainableParams();
        if (!jd.hasTrainableParams()) return;
        if (jac.size() != tp.size())
            throw LightningException("The size of preallocated jacobian must be same as the number of trainable parameters.");
        std::unique_ptr<StateVectorT> owned;
        const StateVectorT *sv = device_psi;
        if (!sv) {
            owned = std::make_unique<StateVectorT>(jd.getPtrStateVec(), jd.getSizeStateVec());
            sv = owned.get();
        }
        const auto &ops = jd.getOperations();
        std::vector<b200sv_op> cops(ops.getSize());
        std::vector<std::vector<uint32_t>> w(ops.getSize());
        std::vector<std::vector<double>> p(ops.getSize());
        for (size_t i = 0; i < ops.getSize(); ++i) {
            w[i].assign(ops.getOpsWires()[i].begin(), ops.getOpsWires()[i].end());
            p[i].assign(ops.getOpsParams()[i].begin(), ops.getOpsParams()[i].end());
            const bool has_mat = !ops.getOpsMatrices()[i].empty();
            cops[i] = b200sv_op{has_mat ? (uint32_t)B200SV_OP_MATRIX : op_id(ops.getOpsName()[i]), (uint32_t)w[i].size(),
                                w[i].data(), ops.getOpsInverses()[i] ? 1 : 0, (uint32_t)p[i].size(), p[i].data(),
                                has_mat ? ops.getOpsMatrices()[i].data() : nullptr};
        }
        std::vector<uint64_t> tpu(tp.begin(), tp.end());
        std::vector<double> out(2 * tp.size());
        check(b200sv_vjp_state(sv->handle(), cops.data(), (uint32_t)cops.size(), dy.data(), dy.size(), tpu.data(),
                               (uint32_t)tpu.size(), apply_operations ? 1 : 0, out.data()));
        for (size_t j = 0; j < tp.size(); ++j) jac[j] = ComplexT((PrecisionT)out[2 * j], (PrecisionT)out[2 * j + 1]);
    }
};

}  // namespace Pennylane::LightningB200
