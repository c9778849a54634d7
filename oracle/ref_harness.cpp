// ref_harness.cpp — extern "C" access to the reference's own FalconnPP class
// (src/FalconnPP.{h,cpp}, compiled unchanged from the reference tree against
// the Eigen/Boost subset in oracle/shim/).  TEST INFRASTRUCTURE ONLY: the
// tests use it to pin the oracle and the GPU path to the reference's code,
// and bench.py's reference arm times it on the host cores.  Nothing in the
// product links it.
//
// The index internals the reference keeps protected (vecPair_BucketPos,
// vecTables_1D, vecTables_2D, matrix_X, bitHD1/2, fhtDim) are read through a
// derived class; the calls themselves are the reference's build2Layers_1D /
// query2Layers_1D / build2Layers / query2Layers (src/FalconnPP.cpp:21-707,
// :722-1413) and Index2Layers / set_qProbes / set_threads
// (src/FalconnPP.h:85-123).
#include <stdint.h>

#include <vector>

#include "FalconnPP.h"

namespace {

struct RefIndex : public FalconnPP {
  RefIndex(int n, int d) : FalconnPP(n, d) {}
  const std::vector<std::pair<uint32_t, uint16_t>>& pos() const { return vecPair_BucketPos; }
  const IVector& ids() const { return vecTables_1D; }
  const std::vector<IVector>& tables2d() const { return vecTables_2D; }
  const MatrixXf& X() const { return matrix_X; }
  const boost::dynamic_bitset<>& b1() const { return bitHD1; }
  const boost::dynamic_bitset<>& b2() const { return bitHD2; }
  int fht() const { return fhtDim; }
  // adopt an index built elsewhere (the GPU's): centred rows, sign bits,
  // CSR bucket offsets (bucket order) and ids, in the reference's members
  void adopt(const float* Xc, const uint8_t* b1, const uint8_t* b2, long long nbits, const uint32_t* start,
             long long nb, const int32_t* ids, long long nids) {
    matrix_X = MatrixXf::Zero(n_features, n_points);
    for (long j = 0; j < n_points; ++j)
      for (long i = 0; i < n_features; ++i) matrix_X(i, j) = Xc[(size_t)j * n_features + i];
    bitHD1 = boost::dynamic_bitset<>(nbits);
    bitHD2 = boost::dynamic_bitset<>(nbits);
    for (long long i = 0; i < nbits; ++i) {
      bitHD1[i] = b1[i] != 0;
      bitHD2[i] = b2[i] != 0;
    }
    vecPair_BucketPos.assign(nb, std::make_pair(0u, (uint16_t)0));
    for (long long b = 0; b < nb; ++b) vecPair_BucketPos[b] = std::make_pair(start[b], (uint16_t)(start[b + 1] - start[b]));
    vecTables_1D.assign(ids, ids + nids);
  }
  int points() const { return n_points; }
  int features() const { return n_features; }
};

}  // namespace

extern "C" {

void* ref_create(int n, int d) { return new RefIndex(n, d); }

void ref_destroy(void* h) { delete static_cast<RefIndex*>(h); }

void ref_set_index_param(void* h, int L, int D, int bucket_minSize, float alpha, int iProbes, int n_threads,
                         int seed) {
  static_cast<RefIndex*>(h)->Index2Layers(L, D, bucket_minSize, alpha, iProbes, n_threads, seed);
}

void ref_set_qprobes(void* h, int q) { static_cast<RefIndex*>(h)->set_qProbes(q); }

void ref_set_threads(void* h, int t) { static_cast<RefIndex*>(h)->set_threads(t); }

// X: n points of d floats (the d x n column-major matrix the reference takes)
void ref_build(void* h, const float* X, int two_d) {
  RefIndex* r = static_cast<RefIndex*>(h);
  Map<const MatrixXf> m(X, r->features(), r->points());
  if (two_d)
    r->build2Layers(m);
  else
    r->build2Layers_1D(m);
}

// Q: nq queries of d floats; out: nq x k int32 (the Q x k matrix returned)
void ref_query(void* h, const float* Q, int nq, int k, int verbose, int two_d, int32_t* out) {
  RefIndex* r = static_cast<RefIndex*>(h);
  Map<const MatrixXf> m(Q, r->features(), nq);
  MatrixXi res = two_d ? r->query2Layers(m, k, verbose != 0) : r->query2Layers_1D(m, k, verbose != 0);
  for (int q = 0; q < nq; ++q)
    for (int j = 0; j < k; ++j) out[(size_t)q * k + j] = res(q, j);
}

// adopt an index built elsewhere; the buckets must hold at most 65535 ids
// (the reference's uint16 sizes)
void ref_import(void* h, const float* Xc, const uint8_t* b1, const uint8_t* b2, long long nbits,
                const uint32_t* start, long long nb, const int32_t* ids, long long nids) {
  static_cast<RefIndex*>(h)->adopt(Xc, b1, b2, nbits, start, nb, ids, nids);
}

int ref_fht_dim(void* h) { return static_cast<RefIndex*>(h)->fht(); }

long long ref_num_ids(void* h) { return (long long)static_cast<RefIndex*>(h)->ids().size(); }

long long ref_num_buckets(void* h) { return (long long)static_cast<RefIndex*>(h)->pos().size(); }

// the 1D layout: per bucket (position, uint16 size), and the id array
void ref_get_tables(void* h, uint32_t* pos, uint16_t* size, int32_t* ids) {
  const RefIndex* r = static_cast<RefIndex*>(h);
  const auto& p = r->pos();
  for (size_t i = 0; i < p.size(); ++i) {
    pos[i] = p[i].first;
    size[i] = p[i].second;
  }
  const IVector& v = r->ids();
  for (size_t i = 0; i < v.size(); ++i) ids[i] = v[i];
}

// the 2D layout: bucket sizes, then the buckets concatenated in bucket order
long long ref_num_ids_2d(void* h) {
  long long t = 0;
  for (const auto& b : static_cast<RefIndex*>(h)->tables2d()) t += (long long)b.size();
  return t;
}

void ref_get_tables_2d(void* h, uint32_t* size, int32_t* ids) {
  const auto& t = static_cast<RefIndex*>(h)->tables2d();
  size_t o = 0;
  for (size_t i = 0; i < t.size(); ++i) {
    size[i] = (uint32_t)t[i].size();
    for (int id : t[i]) ids[o++] = id;
  }
}

// the centred data the reference stores (n points of d floats)
void ref_get_centered(void* h, float* Xc) {
  const MatrixXf& X = static_cast<RefIndex*>(h)->X();
  for (long j = 0; j < X.cols(); ++j)
    for (long i = 0; i < X.rows(); ++i) Xc[(size_t)j * X.rows() + i] = X(i, j);
}

void ref_get_bits(void* h, uint8_t* b1, uint8_t* b2) {
  const RefIndex* r = static_cast<RefIndex*>(h);
  for (size_t i = 0; i < r->b1().size(); ++i) {
    b1[i] = r->b1()[i] ? 1 : 0;
    b2[i] = r->b2()[i] ? 1 : 0;
  }
}

}  // extern "C"
