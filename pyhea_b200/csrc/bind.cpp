// bind.cpp -- pybind11 module `accelerate`, the drop-in for pyhea.cpp.accelerate.
//
// Same names, argument order and return types as pyhea/cpp/bind.cpp:7-120:
//   run_local_parallel_hcs_cuda(nnet, step, task, depth, thr, nbor, element,
//                               weight, target_sro) -> (list[list[int]], list[float])
//   cuda_available() -> bool
//   run_local_parallel_hcs(...)  (the CPU engine, bind.cpp:7-46) is not part of
//                               this module and raises RuntimeError
// It calls the C ABI of libhea_cuda.so (include/hea_cuda.h) and nothing else;
// the GIL is released while the search runs.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cstdint>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "hea_cuda.h"

namespace py = pybind11;

namespace {

[[noreturn]] void raise_for(int rc)
{
    std::string msg = hea_last_error();
    if (rc == HEA_ERR_INVALID) throw py::value_error(msg);
    throw std::runtime_error(msg);
}

// One shell of one site: a numpy integer array or any sequence of ints.
void append_shell(const py::handle &shell, std::vector<int32_t> &out)
{
    if (py::isinstance<py::array>(shell)) {
        auto a = py::array_t<int64_t, py::array::c_style | py::array::forcecast>::ensure(shell);
        if (!a) throw py::value_error("nbor shells must hold integers");
        const int64_t *p = a.data();
        for (py::ssize_t i = 0; i < a.size(); ++i) {
            if (p[i] < INT32_MIN || p[i] > INT32_MAX) throw py::value_error("neighbour id out of int32 range");
            out.push_back((int32_t)p[i]);
        }
        return;
    }
    for (const py::handle &v : py::reinterpret_borrow<py::sequence>(shell)) out.push_back(py::cast<int32_t>(v));
}

// Flatten nbor[N][>=S][Z_k] to [N][sum Z] using the first S shells
// (accelerate.cu:1132-1144); every site must have the same shell sizes.
void flatten_nbor(const py::handle &nbor, int S, int N, std::vector<int32_t> &flat, std::vector<int32_t> &sizes)
{
    auto sites = py::reinterpret_borrow<py::sequence>(nbor);
    if ((int64_t)py::len(sites) != N)
        throw py::value_error("nbor lists " + std::to_string(py::len(sites)) + " sites but element sums to " +
                              std::to_string(N));
    sizes.assign(S, -1);
    for (int s = 0; s < N; ++s) {
        if (s == 1) flat.reserve((size_t)N * flat.size());
        auto shells = py::reinterpret_borrow<py::sequence>(sites[s]);
        if ((int)py::len(shells) < S)
            throw py::value_error("site " + std::to_string(s) + " has " + std::to_string(py::len(shells)) +
                                  " shells; weight asks for " + std::to_string(S));
        for (int k = 0; k < S; ++k) {
            const size_t before = flat.size();
            append_shell(shells[k], flat);
            const int z = (int)(flat.size() - before);
            if (sizes[k] < 0) {
                sizes[k] = z;
            } else if (z != sizes[k]) {
                throw py::value_error("shell " + std::to_string(k) + " of site " + std::to_string(s) + " has " +
                                      std::to_string(z) + " neighbours, site 0 has " + std::to_string(sizes[k]) +
                                      "; shells must have one size for all sites");
            }
        }
    }
}

py::tuple run_cuda(int nnet, int step, int task, int depth, double thr, const py::object &nbor,
                   const std::vector<int> &element, const std::vector<double> &weight, const py::object &target_sro,
                   const py::object &seed, bool verbose)
{
    const int T = (int)element.size(), S = (int)weight.size();
    int64_t n64 = 0;
    for (int v : element) n64 += v;
    if (T < 1 || S < 1) throw py::value_error("element and weight must not be empty");
    if (n64 < 1 || n64 > INT32_MAX / 2) throw py::value_error("element counts must sum to a positive site count");
    const int N = (int)n64;

    std::vector<int32_t> flat, sizes;
    flatten_nbor(nbor, S, N, flat, sizes);

    auto rows = py::reinterpret_borrow<py::sequence>(target_sro);
    if ((int)py::len(rows) < S)
        throw py::value_error("target_sro has " + std::to_string(py::len(rows)) + " shells; weight asks for " +
                              std::to_string(S));
    std::vector<double> target;
    for (int k = 0; k < S; ++k) {
        std::vector<double> r = py::cast<std::vector<double>>(rows[k]);
        if ((int)r.size() != T * T)
            throw py::value_error("target_sro shell " + std::to_string(k) + " has " + std::to_string(r.size()) +
                                  " values; expected " + std::to_string(T * T));
        target.insert(target.end(), r.begin(), r.end());
    }
    std::vector<int32_t> species(element.begin(), element.end());

    hea_problem pb{};
    pb.num_sites = N;
    pb.num_types = T;
    pb.num_shells = S;
    pb.shell_sizes = sizes.data();
    pb.nbor = flat.data();
    pb.species = species.data();
    pb.weight = weight.data();
    pb.target_sro = target.data();

    hea_params pr{};
    pr.num_solutions = nnet;
    pr.total_iter = step;
    pr.parallel_task = task;
    pr.converge_depth = depth;
    pr.threshold = thr;
    if (seed.is_none()) {
        std::random_device rd;
        pr.seed = ((uint64_t)rd() << 32) ^ (uint64_t)rd();
    } else {
        pr.seed = py::cast<uint64_t>(seed);
    }
    pr.flags = verbose ? HEA_FLAG_LOG_ITERS : 0;

    std::vector<uint8_t> occ((size_t)nnet > 0 ? (size_t)nnet * N : 0);
    std::vector<double> fit(nnet > 0 ? nnet : 0);
    int rc;
    {
        py::gil_scoped_release release;
        rc = hea_run_local_parallel_hcs(&pb, &pr, occ.data(), fit.data(), nullptr);
    }
    if (rc != HEA_OK) raise_for(rc);

    // rows of Python ints built with the C API: one int object per species
    // value (CPython's cached small ints), a new reference stored per element
    std::vector<py::object> value(256);
    for (int v = 0; v < 256; ++v) value[v] = py::int_(v);
    py::list latts(nnet);
    for (int p = 0; p < nnet; ++p) {
        PyObject *row = PyList_New(N);
        if (!row) throw py::error_already_set();
        const uint8_t *o = occ.data() + (size_t)p * N;
        for (int s = 0; s < N; ++s) {
            PyObject *x = value[o[s]].ptr();
            Py_INCREF(x);
            PyList_SET_ITEM(row, s, x);  // steals the reference
        }
        latts[p] = py::reinterpret_steal<py::list>(row);
    }
    py::list fits(nnet);
    for (int p = 0; p < nnet; ++p) fits[p] = py::float_(fit[p]);
    return py::make_tuple(latts, fits);
}

}  // namespace

PYBIND11_MODULE(accelerate, m)
{
    m.doc() = "B200 swap-search engine with the interface of pyhea.cpp.accelerate";
    m.def("run_local_parallel_hcs_cuda", &run_cuda, py::arg("nnet"), py::arg("step"), py::arg("task"),
          py::arg("depth"), py::arg("thr"), py::arg("nbor"), py::arg("element"), py::arg("weight"),
          py::arg("target_sro"), py::kw_only(), py::arg("seed") = py::none(), py::arg("verbose") = true,
          R"pbdoc(
            Run the local parallel hybrid cuckoo search on the GPU.

            nnet: population size; step: global iterations; task: proposals per
            round; depth: rounds without improvement that end a local search;
            thr: accepted and unused (as in PyHEA); nbor[N][shell][k]: neighbour
            ids; element: atoms per species; weight: shell weights (their number
            selects the shells); target_sro[shell][T*T]: target alpha.
            seed (keyword, optional): fixes every random draw; a fresh seed per
            call when omitted.  verbose: print the per-iteration best fitness.

            Returns (lattices [nnet][N] species ids, fitness [nnet]) ascending.
        )pbdoc");
    m.def("cuda_available", []() { return hea_cuda_available() != 0; },
          "True when a CUDA device is usable (pyhea/cpp/accelerate.cu:33-37).");
    m.def(
        "run_local_parallel_hcs",
        [](py::args, py::kwargs) -> py::tuple {
            throw std::runtime_error(
                "this accelerate module is the B200 GPU engine; the CPU engine (device: cpu) is not part of it. "
                "Use run_local_parallel_hcs_cuda (device: gpu).");
        },
        "Not provided by this module: the CPU engine of pyhea.cpp.accelerate.");
}
