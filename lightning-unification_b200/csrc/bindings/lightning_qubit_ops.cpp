// lightning_qubit_ops.cpp — pybind11 module with the Python surface of the
// reference's lightning_qubit_ops (CS/bindings/Bindings.cpp:39-57,
// CS/bindings/Bindings.hpp:99-614, LQ/bindings/LQubitBindings.hpp:45-264,
// CS/bindings/BindingsBase.hpp:57-82), backed by libb200sv through the C++
// host API.
//
// StateVectorC64/C128(ndarray) borrow the array as the reference does; the
// amplitudes are uploaded to the device, gates run there, and the array is
// written back when the wrapper is released or on sync() — so code that relies
// on the reference's in-place mutation of the array keeps working.
#include <pybind11/complex.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cuda_runtime_api.h>

#include <cstdlib>
#include <sstream>

#include "AdjointJacobianB200.hpp"
#include "MeasurementsB200.hpp"

namespace py = pybind11;
using namespace Pennylane::LightningB200;

namespace {

// CPU memory-model enum of the reference (CS/utils/CPUMemoryModel.hpp:46); the
// device owns the amplitudes here, so host alignment only matters for copies.
enum class CPUMemoryModel : int { Unaligned = 0, Aligned256 = 1, Aligned512 = 2 };

template <class T> class PySV {
  public:
    using PrecisionT = T;
    using ComplexT = std::complex<T>;
    StateVectorB200<T> sv;
    py::array_t<ComplexT> borrowed;
    bool dirty = false;

    explicit PySV(const py::array_t<ComplexT> &arr) : sv(check_len(arr)), borrowed(arr) {
        sv.updateData(static_cast<const ComplexT *>(arr.request().ptr), (size_t)arr.request().shape[0]);
    }
    ~PySV() {
        if (dirty && borrowed) {
            try {
                sync();
            } catch (...) {
            }
        }
    }
    static size_t check_len(const py::array_t<ComplexT> &arr) {
        auto info = arr.request();
        if (info.ndim != 1) throw std::invalid_argument("NumPy array must be a 1-dimensional array");
        if (info.itemsize != (py::ssize_t)sizeof(ComplexT))
            throw std::invalid_argument("NumPy array must be of type np.complex64 or np.complex128");
        size_t n = 0, len = (size_t)info.shape[0];
        while ((size_t(1) << n) < len) ++n;
        if ((size_t(1) << n) != len || len < 2) throw std::invalid_argument("The length of the array must be 2^n");
        return n;
    }
    void sync() {
        auto info = borrowed.request(true);
        sv.getData(static_cast<ComplexT *>(info.ptr), (size_t)info.shape[0]);
        dirty = false;
    }
};

template <class T> void register_precision(py::module_ &m, py::module_ &obsm, py::module_ &algm) {
    using SV = StateVectorB200<T>;
    using W = PySV<T>;
    using ComplexT = std::complex<T>;
    using np_c = py::array_t<ComplexT, py::array::c_style | py::array::forcecast>;
    using np_r = py::array_t<T, py::array::c_style | py::array::forcecast>;
    const std::string bits = std::to_string(sizeof(ComplexT) * 8);

    // ---- StateVectorC* --------------------------------------------------------
    auto cls = py::class_<W>(m, ("StateVectorC" + bits).c_str(), py::module_local());
    cls.def(py::init([](const py::array_t<ComplexT> &a) { return new W(a); }), py::keep_alive<1, 2>());
    cls.def_property_readonly("size", [](const W &w) { return w.sv.getLength(); });
    for (const auto &name : gate_names()) {
        cls.def(
            name.c_str(),
            [name](W &w, const std::vector<size_t> &wires, bool inverse, const std::vector<T> &params) {
                w.sv.applyOperation(name, wires, inverse, params);
                w.dirty = true;
            },
            ("Apply the " + name + " gate.").c_str());
    }
    cls.def("applyMatrix",
            [](W &w, const np_c &matrix, const std::vector<size_t> &wires, bool inverse) {
                auto b = matrix.request();
                w.sv.applyMatrix(std::vector<ComplexT>(static_cast<const ComplexT *>(b.ptr),
                                                       static_cast<const ComplexT *>(b.ptr) + b.size),
                                 wires, inverse);
                w.dirty = true;
            },
            "Apply a given matrix to wires.");
    cls.def("kernel_map", [](const W &) {
        py::dict d;
        for (const auto &n : gate_names()) d[n.c_str()] = "B200";
        for (const auto &[n, id] : generator_ids()) d[("Generator" + n).c_str()] = "B200";
        for (const char *n : {"SingleQubitOp", "TwoQubitOp", "MultiQubitOp"}) d[n] = "B200";
        return d;
    });
    cls.def("sync", &W::sync, "Write the device amplitudes back into the borrowed array.");
    cls.def("DeviceToHost", [](W &w, py::array_t<ComplexT> &out) {
        auto b = out.request(true);
        w.sv.getData(static_cast<ComplexT *>(b.ptr), (size_t)b.shape[0]);
    });
    cls.def("HostToDevice", [](W &w, const np_c &in) {
        auto b = in.request();
        w.sv.updateData(static_cast<const ComplexT *>(b.ptr), (size_t)b.shape[0]);
        w.dirty = true;
    });
    cls.def("resetStateVector", [](W &w) {
        w.sv.resetStateVector();
        w.dirty = true;
    });
    cls.def("setBasisState", [](W &w, size_t index) {
        w.sv.setBasisState(index);
        w.dirty = true;
    });
    cls.def("applyGenerator", [](W &w, const std::string &name, const std::vector<size_t> &wires, bool adj) {
        w.dirty = true;
        return w.sv.applyGenerator(name, wires, adj);
    });

    // ---- observables ------------------------------------------------------------
    using Obs = Observable<SV>;
    py::class_<Obs, std::shared_ptr<Obs>>(obsm, ("ObservableC" + bits).c_str(), py::module_local());
    auto eq = [](const Obs &a, py::handle b) {
        if (!py::isinstance<Obs>(b)) return false;
        return a == *b.cast<std::shared_ptr<Obs>>();
    };
    py::class_<NamedObs<SV>, std::shared_ptr<NamedObs<SV>>, Obs>(obsm, ("NamedObsC" + bits).c_str(), py::module_local())
        .def(py::init([](const std::string &n, const std::vector<size_t> &w) { return NamedObs<SV>(n, w); }))
        .def("__repr__", &NamedObs<SV>::getObsName)
        .def("get_wires", &NamedObs<SV>::getWires)
        .def("__eq__", eq);
    py::class_<HermitianObs<SV>, std::shared_ptr<HermitianObs<SV>>, Obs>(obsm, ("HermitianObsC" + bits).c_str(),
                                                                       py::module_local())
        .def(py::init([](const np_c &mat, const std::vector<size_t> &w) {
            auto b = mat.request();
            const auto *p = static_cast<const ComplexT *>(b.ptr);
            return HermitianObs<SV>(std::vector<ComplexT>(p, p + b.size), w);
        }))
        .def("__repr__", &HermitianObs<SV>::getObsName)
        .def("get_wires", &HermitianObs<SV>::getWires)
        .def("__eq__", eq);
    py::class_<TensorProdObs<SV>, std::shared_ptr<TensorProdObs<SV>>, Obs>(obsm, ("TensorProdObsC" + bits).c_str(),
                                                                         py::module_local())
        .def(py::init([](const std::vector<std::shared_ptr<Obs>> &o) { return TensorProdObs<SV>(o); }))
        .def("__repr__", &TensorProdObs<SV>::getObsName)
        .def("get_wires", &TensorProdObs<SV>::getWires)
        .def("__eq__", eq);
    py::class_<Hamiltonian<SV>, std::shared_ptr<Hamiltonian<SV>>, Obs>(obsm, ("HamiltonianC" + bits).c_str(),
                                                                     py::module_local())
        .def(py::init([](const np_r &coeffs, const std::vector<std::shared_ptr<Obs>> &o) {
            auto b = coeffs.request();
            const auto *p = static_cast<const T *>(b.ptr);
            return Hamiltonian<SV>(std::vector<T>(p, p + b.size), o);
        }))
        .def("__repr__", &Hamiltonian<SV>::getObsName)
        .def("get_wires", &Hamiltonian<SV>::getWires)
        .def("__eq__", eq);

    // ---- MeasurementsC* -------------------------------------------------------
    using M = Measurements<SV>;
    // LQ/bindings/LQubitBindings.hpp:112-118: size_t indices, values in the state's precision
    using SparseIdx = py::array_t<size_t, py::array::c_style | py::array::forcecast>;
    using ArrC = py::array_t<std::complex<T>, py::array::c_style | py::array::forcecast>;
    auto sv_of = [](W &w) -> const SV & { return w.sv; };
    (void)sv_of;
    py::class_<M>(m, ("MeasurementsC" + bits).c_str(), py::module_local())
        .def(py::init([](W &w) { return new M(w.sv); }), py::keep_alive<1, 2>())
        .def("probs", [](M &ms, const std::vector<size_t> &w) { return py::array_t<T>(py::cast(ms.probs(w))); })
        .def("probs", [](M &ms) { return py::array_t<T>(py::cast(ms.probs())); })
        .def("expval", [](M &ms, const std::shared_ptr<Obs> &o) { return ms.expval(*o); },
             "Expected value of an observable object.")
        .def("expval", [](M &ms, const std::string &name, const std::vector<size_t> &w) { return ms.expval(name, w); },
             "Expected value of an operation by name.")
        .def(
            "expval",
            [](M &ms, const SparseIdx &row_map, const SparseIdx &entries, const ArrC &values) {
                return ms.expval(row_map.data(), (size_t)row_map.size(), entries.data(), values.data(),
                                 (size_t)values.size());
            },
            "Expected value of a sparse Hamiltonian.")
        .def("var", [](M &ms, const std::shared_ptr<Obs> &o) { return ms.var(*o); })
        .def("var", [](M &ms, const std::string &name, const std::vector<size_t> &w) { return ms.var(name, w); })
        .def(
            "var",
            [](M &ms, const SparseIdx &row_map, const SparseIdx &entries, const ArrC &values) {
                return ms.var(row_map.data(), (size_t)row_map.size(), entries.data(), values.data(),
                              (size_t)values.size());
            },
            "Variance of a sparse Hamiltonian.")
        .def("generate_samples",
             [](M &ms, size_t num_wires, size_t num_shots) {
                 auto r = ms.generate_samples(num_shots);
                 py::array_t<size_t> a({num_shots, num_wires});
                 std::copy(r.begin(), r.end(), a.mutable_data());
                 return a;
             })
        .def("generate_samples",
             [](M &ms, size_t num_wires, size_t num_shots, uint64_t seed) {
                 auto r = ms.generate_samples(num_shots, seed);
                 py::array_t<size_t> a({num_shots, num_wires});
                 std::copy(r.begin(), r.end(), a.mutable_data());
                 return a;
             })
        .def("generate_mcmc_samples",  // LQ/bindings/LQubitBindings.hpp:162-182
             [](M &ms, size_t num_wires, const std::string &kernelname, size_t num_burnin, size_t num_shots) {
                 auto r = ms.generate_samples_metropolis(kernelname, num_burnin, num_shots);
                 py::array_t<size_t> a({num_shots, num_wires});
                 std::copy(r.begin(), r.end(), a.mutable_data());
                 return a;
             })
        .def("generate_mcmc_samples",
             [](M &ms, size_t num_wires, const std::string &kernelname, size_t num_burnin, size_t num_shots,
                uint64_t seed, uint32_t num_chains) {
                 auto r = ms.generate_samples_metropolis(kernelname, num_burnin, num_shots, seed, num_chains);
                 py::array_t<size_t> a({num_shots, num_wires});
                 std::copy(r.begin(), r.end(), a.mutable_data());
                 return a;
             },
             py::arg("num_wires"), py::arg("kernelname"), py::arg("num_burnin"), py::arg("num_shots"),
             py::arg("seed"), py::arg("num_chains") = 4096)
        .def("generate_samples_from_uniforms", [](M &ms, size_t num_wires,
                                                  const py::array_t<double, py::array::c_style | py::array::forcecast> &u) {
            auto b = u.request();
            std::vector<double> uv(static_cast<const double *>(b.ptr), static_cast<const double *>(b.ptr) + b.size);
            auto r = ms.generate_samples_from_uniforms(uv);
            py::array_t<size_t> a({(size_t)uv.size(), num_wires});
            std::copy(r.begin(), r.end(), a.mutable_data());
            return a;
        });

    // ---- algorithms ---------------------------------------------------------------
    using Ops = OpsData<SV>;
    py::class_<Ops>(algm, ("OpsStructC" + bits).c_str(), py::module_local())
        .def(py::init<std::vector<std::string>, std::vector<std::vector<T>>, std::vector<std::vector<size_t>>,
                      std::vector<bool>, std::vector<std::vector<ComplexT>>>())
        .def("__repr__", [](const Ops &ops) {
            std::ostringstream s;
            s << "Operations: [";
            for (size_t i = 0; i < ops.getSize(); ++i) {
                s << "{'name': " << ops.getOpsName()[i] << ", 'params': [";
                for (size_t j = 0; j < ops.getOpsParams()[i].size(); ++j) s << (j ? ", " : "") << ops.getOpsParams()[i][j];
                s << "], 'inv': " << (ops.getOpsInverses()[i] ? 1 : 0) << "}" << (i + 1 < ops.getSize() ? "," : "");
            }
            s << "]";
            return s.str();
        });
    algm.def(("create_ops_listC" + bits).c_str(),
             [](const std::vector<std::string> &names, const std::vector<std::vector<T>> &params,
                const std::vector<std::vector<size_t>> &wires, const std::vector<bool> &inv,
                const std::vector<np_c> &mats) {
                 std::vector<std::vector<ComplexT>> cm(names.size());
                 for (size_t i = 0; i < names.size() && i < mats.size(); ++i) {
                     auto b = mats[i].request();
                     if (b.size) {
                         const auto *p = static_cast<const ComplexT *>(b.ptr);
                         cm[i].assign(p, p + b.size);
                     }
                 }
                 return Ops(names, params, wires, inv, cm);
             });
    py::class_<AdjointJacobian<SV>>(algm, ("AdjointJacobianC" + bits).c_str(), py::module_local())
        .def(py::init<>())
        .def("__call__", [](AdjointJacobian<SV> &adj, W &w, const std::vector<std::shared_ptr<Obs>> &obs,
                            const Ops &ops, const std::vector<size_t> &tp) {
            std::vector<T> jac(obs.size() * tp.size(), T{0});
            JacobianData<SV> jd(ops.getTotalNumParams(), w.sv.getLength(), nullptr, obs, ops, tp);
            adj.adjointJacobian(std::span<T>(jac), jd, false, &w.sv);
            return py::array_t<T>(py::cast(jac));
        });
    py::class_<VectorJacobianProduct<SV>>(algm, ("VectorJacobianProductC" + bits).c_str(), py::module_local())
        .def(py::init<>())
        .def("__call__", [](VectorJacobianProduct<SV> &vjp, W &w, const Ops &ops, const py::array_t<ComplexT> &dy,
                            const std::vector<size_t> &tp) {
            auto b = dy.request();
            std::vector<ComplexT> jac(tp.size(), ComplexT{0, 0});
            JacobianData<SV> jd(ops.getTotalNumParams(), w.sv.getLength(), nullptr, {}, ops, tp);
            vjp(std::span<ComplexT>(jac), jd,
                std::span<const ComplexT>(static_cast<const ComplexT *>(b.ptr), (size_t)b.size), false, &w.sv);
            return py::array_t<ComplexT>(py::cast(jac));
        });
}

}  // namespace

PYBIND11_MODULE(lightning_qubit_ops, m) {
    m.doc() = "lightning.qubit operations on the B200 state-vector engine (libb200sv)";
    py::enum_<CPUMemoryModel>(m, "CPUMemoryModel", py::module_local())
        .value("Unaligned", CPUMemoryModel::Unaligned)
        .value("Aligned256", CPUMemoryModel::Aligned256)
        .value("Aligned512", CPUMemoryModel::Aligned512);
    m.def("compile_info", [] {
        py::dict d;
        d["cpu.arch"] = "x86_64";
        d["compiler.name"] = "NVCC";
        d["compiler.version"] = std::to_string(__GNUC__) + "." + std::to_string(__GNUC_MINOR__);
        d["AVX2"] = false;
        d["AVX512F"] = false;
        d["CUDA.arch"] = "sm_100a";
        return d;
    });
    m.def("runtime_info", [] {
        py::dict d;
        int n = 0;
        b200sv_device_count(&n);
        d["CUDA.devices"] = n;
        int rt = 0;
        cudaRuntimeGetVersion(&rt);
        d["CUDA.runtime"] = rt;
        return d;
    });
    m.def("backend_info", [] {
        py::dict d;
        d["NAME"] = "lightning.qubit";
        d["DEVICE"] = "B200";
        return d;
    });
    m.def("get_alignment", [](const py::array &a) {
        const auto p = reinterpret_cast<uintptr_t>(a.request().ptr);
        return (p % 64 == 0) ? CPUMemoryModel::Aligned512 : (p % 32 == 0) ? CPUMemoryModel::Aligned256
                                                                          : CPUMemoryModel::Unaligned;
    });
    m.def("best_alignment", [] { return CPUMemoryModel::Aligned512; });
    m.def("allocate_aligned_array", [](size_t size, const py::dtype &dt) {
        return py::array(dt, {size});
    });
    py::module_ obsm = m.def_submodule("observables", "Submodule for observables classes.");
    py::module_ algm = m.def_submodule("algorithms", "Submodule for the algorithms functionality.");
    register_precision<float>(m, obsm, algm);
    register_precision<double>(m, obsm, algm);
}
