// The C++ host API (StateVectorB200, Measurements, the Observable family,
// AdjointJacobian) driven the way the reference's C++ tests drive lightning.qubit:
// every result is printed as one JSON object per line for tests/test_gpu_host_cpp.py,
// which checks it against the oracle and the reference's known values.
#include <cmath>
#include <complex>
#include <cstdio>
#include <memory>
#include <span>
#include <string>
#include <vector>

#include "AdjointJacobianB200.hpp"
#include "MeasurementsB200.hpp"

using namespace Pennylane::LightningB200;
using SV = StateVectorB200<double>;
using cd = std::complex<double>;

static void print_state(const char *label, const SV &sv) {
    const auto v = sv.getDataVector();
    std::printf("{\"label\": \"%s\", \"re\": [", label);
    for (size_t i = 0; i < v.size(); ++i) std::printf("%s%.17g", i ? ", " : "", v[i].real());
    std::printf("], \"im\": [");
    for (size_t i = 0; i < v.size(); ++i) std::printf("%s%.17g", i ? ", " : "", v[i].imag());
    std::printf("]}\n");
}
static void print_values(const char *label, const std::vector<double> &x) {
    std::printf("{\"label\": \"%s\", \"values\": [", label);
    for (size_t i = 0; i < x.size(); ++i) std::printf("%s%.17g", i ? ", " : "", x[i]);
    std::printf("]}\n");
}

int main() {
    // gates, matrices, generators on 3 qubits (StateVectorBase.hpp:99-194)
    SV sv(3);
    sv.applyOperations({"Hadamard", "RX", "CNOT", "RY", "CRZ"}, {{0}, {1}, {0, 2}, {2}, {1, 0}},
                       {false, false, false, true, false}, {{}, {0.3}, {}, {0.7}, {-1.1}});
    print_state("after_ops", sv);
    const std::vector<cd> u = {cd(0.6, 0.0), cd(0.0, 0.8), cd(0.0, 0.8), cd(0.6, 0.0)};
    sv.applyMatrix(u.data(), {1}, false);
    print_state("after_matrix", sv);
    SV g(sv);
    const double scale = g.applyGenerator("RX", {2}, false);
    print_values("generator_scale", {scale});
    print_state("after_generator", g);

    // measurements (MeasurementsLQubit.hpp:79-372)
    Measurements<SV> m(sv);
    auto pr = m.probs();
    print_values("probs", std::vector<double>(pr.begin(), pr.end()));
    auto pr2 = m.probs({2, 0});
    print_values("probs_20", std::vector<double>(pr2.begin(), pr2.end()));
    print_values("expval_z1", {m.expval("PauliZ", {1})});
    print_values("var_x0", {m.var("PauliX", {0})});
    auto z0 = std::make_shared<NamedObs<SV>>("PauliZ", std::vector<size_t>{0});
    auto x2 = std::make_shared<NamedObs<SV>>("PauliX", std::vector<size_t>{2});
    auto y1 = std::make_shared<NamedObs<SV>>("PauliY", std::vector<size_t>{1});
    auto zx = std::make_shared<TensorProdObs<SV>>(std::vector<std::shared_ptr<Observable<SV>>>{z0, x2});
    Hamiltonian<SV> ham({0.5, -1.25}, {zx, y1});
    print_values("expval_ham", {m.expval(ham)});
    print_values("var_ham", {m.var(ham)});

    // Observable::applyInPlace (Observables.hpp:63-73, ObservablesLQubit.hpp:156-305)
    SV a(sv);
    ham.applyInPlace(a);
    print_state("ham_applied", a);
    SV b(sv);
    zx->applyInPlace(b);
    print_state("zx_applied", b);

    // adjoint Jacobian: RX(p) then <Z> gives -sin(p) (Test_AdjointJacobian.cpp:123-176)
    std::vector<double> jac1;
    for (double p : {-1.2, 0.4, 2.5}) {
        SV s(1);
        s.applyOperation("RX", {0}, false, {p});
        auto data = s.getDataVector();
        OpsData<SV> ops({"RX"}, {{p}}, {{0}}, {false});
        auto z = std::make_shared<NamedObs<SV>>("PauliZ", std::vector<size_t>{0});
        JacobianData<SV> jd(1, data.size(), data.data(), {z}, ops, {0});
        std::vector<double> jac(1);
        AdjointJacobian<SV>().adjointJacobian(std::span<double>(jac), jd);
        jac1.push_back(jac[0]);
    }
    print_values("adjoint_rx_z", jac1);

    // the same 3-qubit circuit differentiated for a Hamiltonian and a named observable
    {
        SV s(3);
        OpsData<SV> ops({"Hadamard", "RX", "CNOT", "RY", "CRZ"}, {{}, {0.3}, {}, {0.7}, {-1.1}},
                        {{0}, {1}, {0, 2}, {2}, {1, 0}}, {false, false, false, true, false});
        s.applyOperations(ops.getOpsName(), ops.getOpsWires(), ops.getOpsInverses(), ops.getOpsParams());
        auto data = s.getDataVector();
        auto hp = std::make_shared<Hamiltonian<SV>>(ham);
        JacobianData<SV> jd(3, data.size(), data.data(), {hp, z0}, ops, {0, 1, 2});
        std::vector<double> jac(6);
        AdjointJacobian<SV>().adjointJacobian(std::span<double>(jac), jd);
        print_values("adjoint_circuit", jac);
    }

    // errors carry the reference's messages (DynamicDispatcher.hpp:322-326)
    try {
        sv.applyOperation("NotAGate", {0});
        print_values("unknown_gate_threw", {0.0});
    } catch (const LightningException &e) {
        std::printf("{\"label\": \"unknown_gate_message\", \"text\": \"%s\"}\n", e.what());
    }
    return 0;
}
