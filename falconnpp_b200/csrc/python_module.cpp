// python_module.cpp — pybind11 module "FalconnPP", class "FalconnPP": the
// reference's Python surface (python/python_wrapper.cpp:14-30) on top of the
// C ABI.  Same method names, keyword names and defaults; inputs are float32
// d x n / d x Q matrices (numpy transposes of (n, d) arrays map without a
// copy, like the reference's Eigen::Ref), query returns an int32 (Q, k) array.
// build2D/query2D produce the same results as build/query in the reference
// (src/FalconnPP.cpp:722-1413), so they run the same GPU path.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <stdexcept>
#include <string>

#include "../../include/falconnpp_b200.h"

namespace py = pybind11;

namespace {

void check(int rc) {
  if (rc == FPP_OK) return;
  const std::string msg = fpp_last_error();
  if (rc == FPP_ERR_INVALID_ARGUMENT) throw py::value_error(msg);
  if (rc == FPP_ERR_OUT_OF_MEMORY) throw std::bad_alloc();
  throw std::runtime_error(msg);
}

using FArray = py::array_t<float, py::array::f_style | py::array::forcecast>;

class FalconnPP {
 public:
  FalconnPP(int n_points, int n_features) : n_(n_points), d_(n_features) {
    check(fpp_create(n_points, n_features, &h_));
  }
  ~FalconnPP() { fpp_destroy(h_); }
  FalconnPP(const FalconnPP&) = delete;
  FalconnPP& operator=(const FalconnPP&) = delete;

  void setIndexParam(int n_tables, int n_proj, int bucket_minSize, float bucket_scale, int iProbes, int n_threads,
                     int random_seed) {
    check(fpp_set_index_param(h_, n_tables, n_proj, bucket_minSize, bucket_scale, iProbes, n_threads, random_seed));
  }
  void set_qProbes(int q) { check(fpp_set_qprobes(h_, q)); }
  void set_threads(int t) { check(fpp_set_threads(h_, t)); }
  void clear() { check(fpp_clear(h_)); }

  void build(const FArray& X) {
    if (X.ndim() != 2 || X.shape(0) != d_ || X.shape(1) != n_)
      throw py::value_error("build: dataset must be a float32 matrix of shape (n_features, n_points)");
    {
      py::gil_scoped_release nogil;
      check(fpp_build(h_, X.data()));
    }
    fpp_print_build_report(h_);
  }

  py::array_t<int32_t> query(const FArray& Q, int k, bool verbose) {
    if (Q.ndim() != 2 || Q.shape(0) != d_)
      throw py::value_error("query: queries must be a float32 matrix of shape (n_features, n_queries)");
    const int nq = (int)Q.shape(1);
    py::array_t<int32_t> out({(py::ssize_t)nq, (py::ssize_t)k});
    int32_t* o = out.mutable_data();
    const float* q = Q.data();
    {
      py::gil_scoped_release nogil;
      check(fpp_query(h_, q, nq, k, verbose ? 1 : 0, o));
    }
    return out;
  }

  // additions (no reference counterpart): persist a built index, and load
  // one saved for the same n_points x n_features
  void save(const std::string& path) { check(fpp_save(h_, path.c_str())); }
  void load(const std::string& path) {
    py::gil_scoped_release nogil;
    check(fpp_load(h_, path.c_str()));
  }

  fpp_index* handle() const { return h_; }

 private:
  fpp_index* h_ = nullptr;
  int n_, d_;
};

}  // namespace

PYBIND11_MODULE(FalconnPP, m) {
  py::class_<FalconnPP>(m, "FalconnPP")
      .def(py::init<const int&, const int&>(), py::arg("n_points"), py::arg("n_features"))
      .def("setIndexParam", &FalconnPP::setIndexParam, py::arg("n_tables"), py::arg("n_proj"),
           py::arg("bucket_minSize"), py::arg("bucket_scale"), py::arg("iProbes"), py::arg("n_threads") = 8,
           py::arg("random_seed") = -1)
      .def("set_qProbes", &FalconnPP::set_qProbes, py::arg("qProbes"))
      .def("set_threads", &FalconnPP::set_threads, py::arg("n_threads"))
      .def("clear", &FalconnPP::clear)
      .def("build2D", &FalconnPP::build, py::arg("dataset"))
      .def("query2D", &FalconnPP::query, py::arg("queries"), py::arg("n_neighbors"), py::arg("verbose") = false)
      .def("build", &FalconnPP::build, py::arg("dataset"))
      .def("query", &FalconnPP::query, py::arg("queries"), py::arg("n_neighbors"), py::arg("verbose") = false)
      .def("save", &FalconnPP::save, py::arg("path"))
      .def("load", &FalconnPP::load, py::arg("path"));
  // the reference's text formats (src/Utilities.cpp:13-61): loadtxtData
  // returns the (n_features, n_points) matrix build() takes; outputFile
  // writes a (Q, k) top-k array one query per line
  m.def(
      "loadtxtData",
      [](const std::string& path, int n_points, int n_features) {
        py::array_t<float, py::array::f_style> X({(py::ssize_t)n_features, (py::ssize_t)n_points});
        check(fpp_load_txt(path.c_str(), n_points, n_features, X.mutable_data(), nullptr));
        return X;
      },
      py::arg("dataset"), py::arg("numPoints"), py::arg("numDim"));
  m.def(
      "outputFile",
      [](const py::array_t<int32_t, py::array::c_style | py::array::forcecast>& topk, const std::string& path) {
        if (topk.ndim() != 2) throw py::value_error("outputFile: top-k must be a (Q, k) int32 array");
        check(fpp_output_file(path.c_str(), topk.data(), (int)topk.shape(0), (int)topk.shape(1)));
      },
      py::arg("matKNN"), py::arg("outputFile"));
}
