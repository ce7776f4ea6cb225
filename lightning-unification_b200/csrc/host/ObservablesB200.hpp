// ObservablesB200.hpp — the Observable hierarchy of lightning.qubit
// (CS/observables/Observables.hpp:35-416, LQ/observables/ObservablesLQubit.hpp:52-356)
// lowered to b200sv_observable records: a list of terms, each a coefficient
// times a tensor product of named or Hermitian factors on disjoint wires.
#pragma once

#include <algorithm>
#include <memory>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "StateVectorB200.hpp"

namespace Pennylane::LightningB200 {

template <class PrecisionT> struct FactorData {
    bool named;
    std::string name;
    std::vector<size_t> wires;
    std::vector<std::complex<PrecisionT>> matrix;
};
template <class PrecisionT> struct TermData {
    double coeff;
    std::vector<FactorData<PrecisionT>> factors;
};

template <class StateVectorT> class Observable {
  public:
    using PrecisionT = typename StateVectorT::PrecisionT;
    virtual ~Observable() = default;
    [[nodiscard]] virtual std::string getObsName() const = 0;
    [[nodiscard]] virtual std::vector<size_t> getWires() const = 0;
    // Terms of this observable (a Hamiltonian has several, the others one).
    [[nodiscard]] virtual std::vector<TermData<PrecisionT>> terms() const = 0;
    [[nodiscard]] bool operator==(const Observable &o) const { return getObsName() == o.getObsName() && same(o); }
    // sv <- O sv (Observables.hpp:63-73; a Hamiltonian sums coeff * term over copies of sv,
    // ObservablesLQubit.hpp:156-305), on the device
    void applyInPlace(StateVectorT &sv) const;

  protected:
    [[nodiscard]] virtual bool same(const Observable &o) const = 0;
};

template <class StateVectorT> class NamedObs final : public Observable<StateVectorT> {
    using PrecisionT = typename StateVectorT::PrecisionT;
    std::string name_;
    std::vector<size_t> wires_;

  public:
    NamedObs(std::string name, std::vector<size_t> wires) : name_(std::move(name)), wires_(std::move(wires)) {
        lookup_gate(name_);
    }
    [[nodiscard]] std::string getObsName() const override {
        std::ostringstream s;
        s << name_ << "[";
        for (size_t i = 0; i < wires_.size(); ++i) s << (i ? ", " : "") << wires_[i];
        s << "]";
        return s.str();
    }
    [[nodiscard]] std::vector<size_t> getWires() const override { return wires_; }
    [[nodiscard]] std::vector<TermData<PrecisionT>> terms() const override {
        return {TermData<PrecisionT>{1.0, {FactorData<PrecisionT>{true, name_, wires_, {}}}}};
    }

  protected:
    [[nodiscard]] bool same(const Observable<StateVectorT> &o) const override {
        auto *p = dynamic_cast<const NamedObs *>(&o);
        return p && p->name_ == name_ && p->wires_ == wires_;
    }
};

template <class StateVectorT> class HermitianObs final : public Observable<StateVectorT> {
    using PrecisionT = typename StateVectorT::PrecisionT;
    std::vector<std::complex<PrecisionT>> matrix_;
    std::vector<size_t> wires_;

  public:
    HermitianObs(std::vector<std::complex<PrecisionT>> m, std::vector<size_t> wires)
        : matrix_(std::move(m)), wires_(std::move(wires)) {
        if (matrix_.size() != (size_t(1) << (2 * wires_.size())))
            throw LightningException("Hermitian matrix size does not match the number of wires");
    }
    [[nodiscard]] std::string getObsName() const override { return "Hermitian"; }
    [[nodiscard]] std::vector<size_t> getWires() const override { return wires_; }
    [[nodiscard]] std::vector<TermData<PrecisionT>> terms() const override {
        return {TermData<PrecisionT>{1.0, {FactorData<PrecisionT>{false, "Hermitian", wires_, matrix_}}}};
    }

  protected:
    [[nodiscard]] bool same(const Observable<StateVectorT> &o) const override {
        auto *p = dynamic_cast<const HermitianObs *>(&o);
        return p && p->matrix_ == matrix_ && p->wires_ == wires_;
    }
};

template <class StateVectorT> class TensorProdObs final : public Observable<StateVectorT> {
    using PrecisionT = typename StateVectorT::PrecisionT;
    std::vector<std::shared_ptr<Observable<StateVectorT>>> obs_;
    std::vector<size_t> all_wires_;

  public:
    explicit TensorProdObs(std::vector<std::shared_ptr<Observable<StateVectorT>>> obs) : obs_(std::move(obs)) {
        std::set<size_t> seen;
        for (auto &o : obs_) {
            if (o->terms().size() != 1) throw LightningException("A tensor product factor must be a single term");
            for (auto w : o->getWires()) {
                if (seen.count(w)) throw LightningException("All wires in observables must be disjoint.");
                seen.insert(w);
            }
        }
        all_wires_.assign(seen.begin(), seen.end());
    }
    [[nodiscard]] std::string getObsName() const override {
        std::string s;
        for (size_t i = 0; i < obs_.size(); ++i) s += (i ? " @ " : "") + obs_[i]->getObsName();
        return s;
    }
    [[nodiscard]] std::vector<size_t> getWires() const override { return all_wires_; }
    [[nodiscard]] std::vector<TermData<PrecisionT>> terms() const override {
        TermData<PrecisionT> t{1.0, {}};
        for (auto &o : obs_) {
            auto sub = o->terms()[0];
            t.coeff *= sub.coeff;
            t.factors.insert(t.factors.end(), sub.factors.begin(), sub.factors.end());
        }
        return {t};
    }

  protected:
    [[nodiscard]] bool same(const Observable<StateVectorT> &o) const override {
        auto *p = dynamic_cast<const TensorProdObs *>(&o);
        if (!p || p->obs_.size() != obs_.size()) return false;
        for (size_t i = 0; i < obs_.size(); ++i)
            if (!(*obs_[i] == *p->obs_[i])) return false;
        return true;
    }
};

template <class StateVectorT> class Hamiltonian final : public Observable<StateVectorT> {
    using PrecisionT = typename StateVectorT::PrecisionT;
    std::vector<PrecisionT> coeffs_;
    std::vector<std::shared_ptr<Observable<StateVectorT>>> obs_;

  public:
    Hamiltonian(std::vector<PrecisionT> coeffs, std::vector<std::shared_ptr<Observable<StateVectorT>>> obs)
        : coeffs_(std::move(coeffs)), obs_(std::move(obs)) {
        if (coeffs_.size() != obs_.size()) throw LightningException("Assertion failed: coeffs_.size() == obs_.size()");
    }
    [[nodiscard]] std::string getObsName() const override {
        std::ostringstream ss;
        ss << "Hamiltonian: { 'coeffs' : [";
        for (size_t i = 0; i < coeffs_.size(); ++i) ss << (i ? ", " : "") << coeffs_[i];
        ss << "], 'observables' : [";
        for (size_t i = 0; i < obs_.size(); ++i) ss << (i ? ", " : "") << obs_[i]->getObsName();
        ss << "]}";
        return ss.str();
    }
    [[nodiscard]] std::vector<size_t> getWires() const override {
        std::set<size_t> w;
        for (auto &o : obs_)
            for (auto x : o->getWires()) w.insert(x);
        return {w.begin(), w.end()};
    }
    [[nodiscard]] std::vector<TermData<PrecisionT>> terms() const override {
        std::vector<TermData<PrecisionT>> r;
        for (size_t i = 0; i < obs_.size(); ++i)
            for (auto t : obs_[i]->terms()) {
                t.coeff *= (double)coeffs_[i];
                r.push_back(std::move(t));
            }
        return r;
    }

  protected:
    [[nodiscard]] bool same(const Observable<StateVectorT> &o) const override {
        auto *p = dynamic_cast<const Hamiltonian *>(&o);
        if (!p || p->coeffs_ != coeffs_ || p->obs_.size() != obs_.size()) return false;
        for (size_t i = 0; i < obs_.size(); ++i)
            if (!(*obs_[i] == *p->obs_[i])) return false;
        return true;
    }
};

// Owns the C records for one observable; valid while alive.
template <class PrecisionT> class ObsRecord {
    std::vector<TermData<PrecisionT>> terms_;
    std::vector<std::vector<uint32_t>> wires_;
    std::vector<std::vector<b200sv_factor>> factors_;
    std::vector<b200sv_term> cterms_;

  public:
    b200sv_observable rec{};
    explicit ObsRecord(std::vector<TermData<PrecisionT>> t) : terms_(std::move(t)) {
        factors_.resize(terms_.size());
        for (size_t i = 0; i < terms_.size(); ++i)
            for (auto &f : terms_[i].factors) wires_.emplace_back(f.wires.begin(), f.wires.end());
        size_t k = 0;
        for (size_t i = 0; i < terms_.size(); ++i) {
            for (auto &f : terms_[i].factors) {
                b200sv_factor bf{};
                bf.kind = f.named ? B200SV_FACTOR_NAMED : B200SV_FACTOR_MATRIX;
                bf.gate = f.named ? lookup_gate(f.name) : 0;
                bf.nwires = (uint32_t)wires_[k].size();
                bf.wires = wires_[k].data();
                bf.matrix = f.named ? nullptr : f.matrix.data();
                factors_[i].push_back(bf);
                ++k;
            }
        }
        for (size_t i = 0; i < terms_.size(); ++i)
            cterms_.push_back(b200sv_term{terms_[i].coeff, (uint32_t)factors_[i].size(), factors_[i].data()});
        rec.nterms = (uint32_t)cterms_.size();
        rec.terms = cterms_.data();
    }
    ObsRecord(const ObsRecord &) = delete;
};

template <class StateVectorT> void Observable<StateVectorT>::applyInPlace(StateVectorT &sv) const {
    ObsRecord<PrecisionT> r(terms());
    check(b200sv_apply_observable(sv.handle(), &r.rec));
}

}  // namespace Pennylane::LightningB200
