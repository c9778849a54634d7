// fpp_persist.cu — saving and loading a built index, and the reference's
// text matrix formats.
//
// The reference rebuilds its index on every run and has no serialisation.
// fpp_save / fpp_load write and read one binary file holding everything the
// query path needs (parameters, sign bits, centre, centred rows, CSR bucket
// offsets and ids), so a server restarts without a rebuild.  fpp_load checks
// the whole file on the host before anything reaches the GPU: ids outside
// [0, n) or offsets out of order would otherwise send the gather kernels to
// addresses outside their buffers.
//
// fpp_load_txt and fpp_output_file read and write the whitespace text
// formats of the reference's loadtxtData and outputFile
// (src/Utilities.cpp:13-61).
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/falconnpp_b200.h"
#include "fpp_handle.h"

namespace {

constexpr char kMagic[8] = {'F', 'P', 'P', 'I', 'D', 'X', '1', '\0'};
constexpr uint32_t kVersion = 1;
constexpr size_t kChunk = 64u << 20;  // bytes staged through the host per copy

// File layout: this header, then the sign bits of both layers (2 x L*3*fhtDim
// bytes, 0/1), the centre (d floats), the centred rows (n x ld floats), the
// CSR offsets (L*4*D^2 + 1 u32) and the ids (n_ids i32), little endian.
struct FileHeader {
  char magic[8];
  uint32_t version;
  uint32_t reserved;
  int32_t n_points, n_features, n_tables, n_proj, bucket_minSize, iProbes, fhtDim, ld;
  float bucket_scale;
  uint32_t max_kept;
  int64_t seed;
  uint64_t n_ids;
  uint64_t n_buckets;
  int64_t n_limited;
  int64_t n_repaired;
  double points_per_table;
};
static_assert(sizeof(FileHeader) == 104, "FileHeader has no padding");

int fail(int code, const std::string& msg) { return fpp::set_last_error(code, msg); }

bool write_all(FILE* f, const void* p, size_t bytes) { return bytes == 0 || fwrite(p, 1, bytes, f) == bytes; }
bool read_all(FILE* f, void* p, size_t bytes) { return bytes == 0 || fread(p, 1, bytes, f) == bytes; }

// device -> file, through a host chunk
bool write_device(FILE* f, const void* dev, size_t bytes, std::vector<unsigned char>& buf) {
  const unsigned char* src = static_cast<const unsigned char*>(dev);
  for (size_t off = 0; off < bytes; off += kChunk) {
    const size_t nb = std::min(kChunk, bytes - off);
    if (cudaMemcpy(buf.data(), src + off, nb, cudaMemcpyDeviceToHost) != cudaSuccess) return false;
    if (!write_all(f, buf.data(), nb)) return false;
  }
  return true;
}

// file -> device, through a host chunk; check(chunk, count) may reject it
template <typename T, typename Check>
bool read_device(FILE* f, T* dev, size_t count, std::vector<unsigned char>& buf, Check check) {
  const size_t per = kChunk / sizeof(T);
  for (size_t off = 0; off < count; off += per) {
    const size_t nc = std::min(per, count - off);
    if (!read_all(f, buf.data(), nc * sizeof(T))) return false;
    if (!check(reinterpret_cast<const T*>(buf.data()), off, nc)) return false;
    if (cudaMemcpy(dev + off, buf.data(), nc * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return false;
  }
  return true;
}

bool is_pow2(int x) { return x > 0 && (x & (x - 1)) == 0; }

}  // namespace

extern "C" {

int fpp_save(fpp_index* h, const char* path) {
  if (!h || !path) return fail(FPP_ERR_INVALID_ARGUMENT, "save: NULL argument");
  std::lock_guard<std::mutex> g(h->mu);
  if (!h->built) return fail(FPP_ERR_NOT_BUILT, "save: the index is not built");
  if (cudaSetDevice(h->device) != cudaSuccess) return fail(FPP_ERR_CUDA, "save: cudaSetDevice failed");
  const fpp::Params& P = h->P;
  const fpp::DeviceIndex& di = h->di;
  FileHeader hd;
  memset(&hd, 0, sizeof(hd));
  memcpy(hd.magic, kMagic, sizeof(kMagic));
  hd.version = kVersion;
  hd.n_points = P.n_points;
  hd.n_features = P.n_features;
  hd.n_tables = P.n_tables;
  hd.n_proj = P.n_proj;
  hd.bucket_minSize = P.bucket_minSize;
  hd.iProbes = P.iProbes;
  hd.fhtDim = P.fhtDim;
  hd.ld = di.ld;
  hd.bucket_scale = P.bucket_scale;
  hd.max_kept = di.max_kept;
  hd.seed = P.seed;
  hd.n_ids = di.n_ids;
  hd.n_buckets = (uint64_t)P.n_tables * 4ull * (uint64_t)P.n_proj * (uint64_t)P.n_proj;
  hd.n_limited = h->bst.n_limited;
  hd.n_repaired = h->bst.n_repaired;
  hd.points_per_table = h->bst.points_per_table;
  const size_t nbits = (size_t)P.n_tables * 3 * P.fhtDim;
  if (h->bits.b1.size() != nbits || h->bits.b2.size() != nbits)
    return fail(FPP_ERR_INVALID_ARGUMENT, "save: the sign bits of the build are missing");
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return fail(FPP_ERR_CUDA, "save: stream failed");
  FILE* f = fopen(path, "wb");
  if (!f) return fail(FPP_ERR_INVALID_ARGUMENT, std::string("save: cannot open ") + path + " for writing");
  std::vector<unsigned char> buf(kChunk);
  bool okw = write_all(f, &hd, sizeof(hd)) && write_all(f, h->bits.b1.data(), nbits) &&
             write_all(f, h->bits.b2.data(), nbits) &&
             write_device(f, di.center, sizeof(float) * (size_t)P.n_features, buf) &&
             write_device(f, di.Xc, sizeof(float) * (size_t)P.n_points * (size_t)di.ld, buf) &&
             write_device(f, di.bucket_off, sizeof(uint32_t) * (size_t)(hd.n_buckets + 1), buf) &&
             write_device(f, di.ids, sizeof(int32_t) * (size_t)di.n_ids, buf);
  okw = (fclose(f) == 0) && okw;
  if (!okw) return fail(FPP_ERR_INVALID_ARGUMENT, std::string("save: writing ") + path + " failed");
  return fpp::clear_last_error();
}

int fpp_load(fpp_index* h, const char* path) {
  if (!h || !path) return fail(FPP_ERR_INVALID_ARGUMENT, "load: NULL argument");
  std::lock_guard<std::mutex> g(h->mu);
  FILE* f = fopen(path, "rb");
  if (!f) return fail(FPP_ERR_INVALID_ARGUMENT, std::string("load: cannot open ") + path);
  auto bad = [&](const std::string& why) {
    fclose(f);
    return fail(FPP_ERR_INVALID_ARGUMENT, std::string("load: ") + path + ": " + why);
  };
  FileHeader hd;
  if (!read_all(f, &hd, sizeof(hd)) || memcmp(hd.magic, kMagic, sizeof(kMagic)) != 0)
    return bad("not an index file of this library");
  if (hd.version != kVersion) return bad("unsupported file version " + std::to_string(hd.version));
  if (hd.n_points != h->P.n_points || hd.n_features != h->P.n_features)
    return bad("the file holds " + std::to_string(hd.n_points) + " x " + std::to_string(hd.n_features) +
               " points, the handle was created for " + std::to_string(h->P.n_points) + " x " +
               std::to_string(h->P.n_features));
  if (hd.n_tables < 1 || !is_pow2(hd.n_proj) || hd.iProbes < 1 || hd.iProbes > hd.n_proj ||
      hd.fhtDim != fpp::derived_fht_dim(hd.n_features, hd.n_proj) || hd.ld != ((hd.n_features + 3) & ~3) ||
      hd.n_buckets != (uint64_t)hd.n_tables * 4ull * (uint64_t)hd.n_proj * (uint64_t)hd.n_proj ||
      hd.n_ids >= (1ull << 32) || hd.n_buckets >= (1ull << 32))
    return bad("inconsistent parameters in the header");
  const size_t nbits = (size_t)hd.n_tables * 3 * hd.fhtDim;
  const unsigned long long expect = sizeof(FileHeader) + 2ull * nbits + 4ull * hd.n_features +
                                    4ull * (unsigned long long)hd.n_points * hd.ld + 4ull * (hd.n_buckets + 1) +
                                    4ull * hd.n_ids;
  if (fseeko(f, 0, SEEK_END) != 0 || (unsigned long long)ftello(f) != expect) return bad("wrong file size");
  if (fseeko(f, sizeof(FileHeader), SEEK_SET) != 0) return bad("seek failed");
  fpp::HostBits bits;
  bits.b1.resize(nbits);
  bits.b2.resize(nbits);
  if (!read_all(f, bits.b1.data(), nbits) || !read_all(f, bits.b2.data(), nbits)) return bad("short read");
  for (size_t i = 0; i < nbits; ++i)
    if (bits.b1[i] > 1 || bits.b2[i] > 1) return bad("sign bits must be 0 or 1");
  if (cudaSetDevice(h->device) != cudaSuccess) {
    fclose(f);
    return fail(FPP_ERR_CUDA, "load: cudaSetDevice failed");
  }
  // the handle's old index goes first; on any failure below it stays unbuilt
  h->ws.release();
  h->bw.release();
    h->bfw.release();
  fpp::free_index(h->di);
  h->built = false;
  fpp::DeviceIndex di;
  di.ld = hd.ld;
  di.n_ids = hd.n_ids;
  std::vector<unsigned char> buf(kChunk);
  const uint64_t n = (uint64_t)hd.n_points;
  uint32_t prev = 0, max_kept = 0;
  bool okr = fpp::dev_malloc(&di.center, sizeof(float) * (size_t)hd.n_features) == cudaSuccess &&
             fpp::dev_malloc(&di.Xc, sizeof(float) * (size_t)n * hd.ld) == cudaSuccess &&
             fpp::dev_malloc(&di.bucket_off, sizeof(uint32_t) * (size_t)(hd.n_buckets + 1)) == cudaSuccess &&
             fpp::dev_malloc(&di.ids, sizeof(int32_t) * std::max<size_t>(1, (size_t)hd.n_ids)) == cudaSuccess;
  std::string why = okr ? "" : "cannot allocate the index on the device";
  auto any = [](const void*, size_t, size_t) { return true; };
  if (okr) okr = read_device(f, di.center, (size_t)hd.n_features, buf, any) &&
                 read_device(f, di.Xc, (size_t)n * hd.ld, buf, any);
  if (okr) {  // offsets: from 0, non-decreasing, ending at n_ids
    okr = read_device(f, di.bucket_off, (size_t)(hd.n_buckets + 1), buf,
                      [&](const uint32_t* c, size_t off, size_t nc) {
                        for (size_t i = 0; i < nc; ++i) {
                          if (off + i == 0 && c[i] != 0u) return false;
                          if (c[i] < prev) return false;
                          if (off + i > 0) max_kept = std::max(max_kept, c[i] - prev);
                          prev = c[i];
                        }
                        return true;
                      });
    if (okr && prev != (uint32_t)hd.n_ids) okr = false;
    if (!okr) why = "bucket offsets out of order or not ending at the id count";
  }
  if (okr) {  // ids in [0, n)
    okr = read_device(f, di.ids, (size_t)hd.n_ids, buf, [&](const int32_t* c, size_t, size_t nc) {
      for (size_t i = 0; i < nc; ++i)
        if (c[i] < 0 || (uint64_t)c[i] >= n) return false;
      return true;
    });
    if (!okr) why = "an id outside [0, n_points)";
  }
  fclose(f);
  fpp::Params P = h->P;
  P.n_tables = hd.n_tables;
  P.n_proj = hd.n_proj;
  P.bucket_minSize = hd.bucket_minSize;
  P.bucket_scale = hd.bucket_scale;
  P.iProbes = hd.iProbes;
  P.seed = hd.seed;
  P.fhtDim = hd.fhtDim;
  fpp::Error err{0, ""};
  if (okr && fpp::upload_flips(P, bits, di, h->stream, err) != fpp::kOk) {
    okr = false;
    why = err.msg;
  }
  if (!okr) {
    fpp::free_index(di);
    return fail(FPP_ERR_INVALID_ARGUMENT, std::string("load: ") + path + ": " + why);
  }
  di.max_kept = max_kept;
  h->P = P;
  h->params_set = true;
  h->bits = std::move(bits);
  h->di = di;
  h->bst = fpp::BuildStats();
  h->bst.n_limited = hd.n_limited;
  h->bst.n_repaired = hd.n_repaired;
  h->bst.points_per_table = hd.points_per_table;
  h->built = true;
  return fpp::clear_last_error();
}

int fpp_load_txt(const char* path, int n_points, int n_features, float* out, long long* n_read) {
  if (!path || !out) return fail(FPP_ERR_INVALID_ARGUMENT, "load_txt: NULL argument");
  if (n_points < 1 || n_features < 1) return fail(FPP_ERR_INVALID_ARGUMENT, "load_txt: sizes must be >= 1");
  FILE* f = fopen(path, "r");
  if (!f) return fail(FPP_ERR_INVALID_ARGUMENT, std::string("load_txt: data file does not exist: ") + path);
  const long long total = (long long)n_points * n_features;
  long long got = 0;
  // each line is one point of n_features values; values the file does not
  // hold stay 0 (the reference's matrix starts zeroed)
  for (long long i = 0; i < total; ++i) {
    float v = 0.0f;
    if (got == i && fscanf(f, "%f", &v) == 1) {
      out[i] = v;
      ++got;
    } else {
      out[i] = 0.0f;
    }
  }
  fclose(f);
  if (n_read) *n_read = got;
  return fpp::clear_last_error();
}

int fpp_output_file(const char* path, const int32_t* topk, int n_queries, int k) {
  if (!path || (!topk && n_queries > 0)) return fail(FPP_ERR_INVALID_ARGUMENT, "output_file: NULL argument");
  if (n_queries < 0 || k < 1) return fail(FPP_ERR_INVALID_ARGUMENT, "output_file: need n_queries >= 0, k >= 1");
  FILE* f = fopen(path, "w");
  if (!f) return fail(FPP_ERR_INVALID_ARGUMENT, std::string("output_file: cannot open ") + path);
  bool okw = true;
  for (int q = 0; q < n_queries && okw; ++q) {  // one query per line, each id followed by a space
    for (int j = 0; j < k && okw; ++j) okw = fprintf(f, "%d ", topk[(size_t)q * k + j]) > 0;
    okw = okw && fputc('\n', f) != EOF;
  }
  okw = (fclose(f) == 0) && okw;
  if (!okw) return fail(FPP_ERR_INVALID_ARGUMENT, std::string("output_file: writing ") + path + " failed");
  return fpp::clear_last_error();
}

}  // extern "C"
