// Output files of the reference model written from device state, formatted on
// the device.
//
// DataOutput (fileio.c:62-122), SubOutput (fileio.c:125-155) and
// writeRestartFile (fileio.c:192-242) write one value per line with
// fprintf("%4.4f \n") (WriteFile, fileio.c:158-181) to
// <saveFolder><name>_<tt>.dat.  Here each value is converted on the GPU with the
// same correctly rounded result as glibc's printf (round to nearest, ties to
// even, on the exact binary value), the lines are packed by an exclusive scan
// of their lengths, and the host only copies the bytes out and writes them.
//
// The conversion is exact for finite |x| < 1e15, where 10^4 |x| fits 64 bits:
// with |x| = m 2^e (m < 2^53), 10^4 |x| = 10^4 m 2^e is formed in 128-bit
// integers and rounded at bit -e.  Any other value (never produced by the model:
// its arrays are elevations, velocities, depths and concentrations) sends the
// whole array to the host's snprintf instead, so the bytes are the same either
// way.
#include <cub/device/device_scan.cuh>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "domain_host.h"
#include "frehd_internal.h"

#define OUT_TRY(expr)                                                                   \
  do {                                                                                  \
    cudaError_t e_ = (expr);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      return frehd::fail(FREHD_ERR_CUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), \
                         __FILE__, __LINE__);                                           \
    }                                                                                   \
  } while (0)

namespace frehd {
namespace {

constexpr int kMaxLine = 32;  // "-999999999999999.9999 \n" is 23 bytes

// "%4.4f \n" of x into out (no terminator); the length, or -1 if x is not finite
// or |x| >= 1e15.
__device__ int fmt_fixed4(double x, char *out) {
  if (!isfinite(x) || fabs(x) >= 1e15) return -1;
  const bool neg = signbit(x);
  unsigned long long bits = __double_as_longlong(fabs(x));
  const int be = (int)(bits >> 52);
  unsigned long long m = bits & ((1ull << 52) - 1);
  int e;
  if (be == 0) {
    e = -1074;  // subnormal
  } else {
    m |= 1ull << 52;
    e = be - 1075;
  }
  unsigned long long R;
  if (m == 0) {
    R = 0;
  } else if (e >= 0) {
    R = (m << e) * 10000ull;  // |x| < 1e15: an exact integer below 2^64
  } else {
    const unsigned __int128 P = (unsigned __int128)m * 10000u;  // < 2^67
    const int s = -e;
    if (s > 68) {
      R = 0;  // P < 2^67 <= 2^(s-2): below half a unit
    } else {
      const unsigned __int128 q = P >> s;
      const unsigned __int128 rem = P - (q << s);
      const unsigned __int128 half = (unsigned __int128)1 << (s - 1);
      R = (unsigned long long)q;
      if (rem > half || (rem == half && (R & 1ull))) ++R;
    }
  }
  const unsigned long long ip = R / 10000ull;
  const unsigned fp = (unsigned)(R % 10000ull);
  char tmp[24];
  int nd = 0;
  unsigned long long v = ip;
  do {
    tmp[nd++] = (char)('0' + (int)(v % 10ull));
    v /= 10ull;
  } while (v);
  int k = 0;
  if (neg) out[k++] = '-';
  while (nd) out[k++] = tmp[--nd];
  out[k++] = '.';
  out[k++] = (char)('0' + fp / 1000);
  out[k++] = (char)('0' + fp / 100 % 10);
  out[k++] = (char)('0' + fp / 10 % 10);
  out[k++] = (char)('0' + fp % 10);
  out[k++] = ' ';
  out[k++] = '\n';
  return k;
}

// Value q of a list: interior cell q of a padded array (minus `sub`), or a raw
// value when the list is given plainly.
struct Values {
  const double *a;  // padded array (pitch > 0) or plain list (pitch == 0)
  int nx, pitch;
  double sub;
  __device__ double at(long q) const {
    if (pitch == 0) return a[q] - sub;
    const int i = (int)(q % nx), j = (int)(q / nx);
    return a[(long)(j + 1) * pitch + (i + kXOff)] - sub;
  }
};

__global__ void k_fmt_len(Values v, long n, unsigned long long *len, int *special) {
  const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (q >= n) return;
  char buf[kMaxLine];
  const int k = fmt_fixed4(v.at(q), buf);
  if (k < 0) {
    atomicOr(special, 1);
    len[q] = 0;
  } else {
    len[q] = (unsigned long long)k;
  }
}

__global__ void k_fmt_write(Values v, long n, const unsigned long long *off, char *out) {
  const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (q >= n) return;
  char buf[kMaxLine];
  const int k = fmt_fixed4(v.at(q), buf);
  char *o = out + off[q];
  for (int c = 0; c < k; ++c) o[c] = buf[c];
}

__global__ void k_gather_values(Values v, long n, double *out) {
  const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (q < n) out[q] = v.at(q);
}

// DataOutput's in-place round trip of the interior surface through the output
// datum (fileio.c:65-66,120-121).
__global__ void k_surf_round_trip(double *s, int nx, int ny, int pitch, double off) {
  const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (q >= (long)nx * ny) return;
  const int i = (int)(q % nx), j = (int)(q / nx);
  double *p = s + (long)(j + 1) * pitch + (i + kXOff);
  const double w = *p - off;
  *p = w + off;
}

// Scratch of one formatting pass, grown as needed.
struct FmtScratch {
  unsigned long long *len = nullptr, *off = nullptr;
  char *text = nullptr;
  void *cub = nullptr;
  int *special = nullptr;
  long cap_n = 0;
  size_t cap_text = 0, cap_cub = 0;
  ~FmtScratch() {
    cudaFree(len);
    cudaFree(off);
    cudaFree(text);
    cudaFree(cub);
    cudaFree(special);
  }
};

int host_format(const std::vector<double> &vals, std::string *s) {
  char line[400];
  s->clear();
  for (double x : vals) {
    const int k = snprintf(line, sizeof(line), "%4.4f \n", x);
    if (k < 0 || k >= (int)sizeof(line)) return fail(FREHD_ERR_INVALID, "value too long to print");
    s->append(line, (size_t)k);
  }
  return FREHD_OK;
}

// Format the n values of v into *s (host bytes).
int format_values(const Values &v, long n, cudaStream_t st, FmtScratch &fs, std::string *s) {
  if (n <= 0) {
    s->clear();
    return FREHD_OK;
  }
  if (n > fs.cap_n) {
    cudaFree(fs.len);
    cudaFree(fs.off);
    fs.len = fs.off = nullptr;
    OUT_TRY(cudaMalloc(&fs.len, sizeof(unsigned long long) * n));
    OUT_TRY(cudaMalloc(&fs.off, sizeof(unsigned long long) * n));
    fs.cap_n = n;
  }
  if (!fs.special) OUT_TRY(cudaMalloc(&fs.special, sizeof(int)));
  OUT_TRY(cudaMemsetAsync(fs.special, 0, sizeof(int), st));
  const unsigned blocks = (unsigned)((n + 255) / 256);
  k_fmt_len<<<blocks, 256, 0, st>>>(v, n, fs.len, fs.special);
  OUT_TRY(cudaGetLastError());
  size_t need = 0;
  OUT_TRY(cub::DeviceScan::ExclusiveSum(nullptr, need, fs.len, fs.off, n, st));
  if (need > fs.cap_cub) {
    cudaFree(fs.cub);
    fs.cub = nullptr;
    OUT_TRY(cudaMalloc(&fs.cub, need));
    fs.cap_cub = need;
  }
  OUT_TRY(cub::DeviceScan::ExclusiveSum(fs.cub, need, fs.len, fs.off, n, st));
  int special = 0;
  unsigned long long last_off = 0, last_len = 0;
  OUT_TRY(cudaMemcpyAsync(&special, fs.special, sizeof(int), cudaMemcpyDeviceToHost, st));
  OUT_TRY(cudaMemcpyAsync(&last_off, fs.off + n - 1, sizeof(last_off), cudaMemcpyDeviceToHost, st));
  OUT_TRY(cudaMemcpyAsync(&last_len, fs.len + n - 1, sizeof(last_len), cudaMemcpyDeviceToHost, st));
  OUT_TRY(cudaStreamSynchronize(st));
  if (special) {  // a value outside the exact device range: print the array on the host
    std::vector<double> h((size_t)n);
    double *dv = nullptr;
    OUT_TRY(cudaMalloc(&dv, sizeof(double) * n));
    k_gather_values<<<blocks, 256, 0, st>>>(v, n, dv);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), dv, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(dv);
    if (e != cudaSuccess) return fail(FREHD_ERR_CUDA, "output gather: %s", cudaGetErrorString(e));
    return host_format(h, s);
  }
  const size_t total = (size_t)(last_off + last_len);
  if (total > fs.cap_text) {
    cudaFree(fs.text);
    fs.text = nullptr;
    OUT_TRY(cudaMalloc(&fs.text, total));
    fs.cap_text = total;
  }
  k_fmt_write<<<blocks, 256, 0, st>>>(v, n, fs.off, fs.text);
  OUT_TRY(cudaGetLastError());
  s->resize(total);
  OUT_TRY(cudaMemcpyAsync(&(*s)[0], fs.text, total, cudaMemcpyDeviceToHost, st));
  OUT_TRY(cudaStreamSynchronize(st));
  return FREHD_OK;
}

int write_file(const char *prefix, const char *name, int tt, const std::string &s) {
  std::string path = std::string(prefix ? prefix : "") + name + "_" + std::to_string(tt) + ".dat";
  FILE *f = fopen(path.c_str(), "w");
  if (!f) return fail(FREHD_ERR_INVALID, "cannot write %s", path.c_str());
  const size_t w = fwrite(s.data(), 1, s.size(), f);
  const int c = fclose(f);
  if (w != s.size() || c != 0) return fail(FREHD_ERR_INVALID, "short write to %s", path.c_str());
  return FREHD_OK;
}

}  // namespace
}  // namespace frehd

using frehd::Values;

extern "C" int frehd_format_fixed4(const double *values, long n, char *out, size_t cap,
                                   size_t *len) {
  if (n < 0 || (n > 0 && !values) || !len) return frehd::fail(FREHD_ERR_INVALID, "bad argument");
  int dev = 0;
  OUT_TRY(cudaGetDevice(&dev));
  double *dv = nullptr;
  if (n > 0) {
    OUT_TRY(cudaMalloc(&dv, sizeof(double) * n));
    cudaError_t e = cudaMemcpy(dv, values, sizeof(double) * n, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFree(dv);
      return frehd::fail(FREHD_ERR_CUDA, "copy: %s", cudaGetErrorString(e));
    }
  }
  std::string s;
  int rc;
  {
    frehd::FmtScratch fs;
    rc = frehd::format_values(Values{dv, 0, 0, 0.0}, n, 0, fs, &s);
  }
  cudaFree(dv);
  if (rc) return rc;
  *len = s.size();
  if (out) {
    if (cap < s.size()) return frehd::fail(FREHD_ERR_INVALID, "output buffer of %zu bytes, %zu needed", cap, s.size());
    memcpy(out, s.data(), s.size());
  }
  return FREHD_OK;
}

extern "C" int frehd_domain_write_output(frehd_domain *d, const char *prefix, int tt, int fields) {
  if (!d || !prefix) return frehd::fail(FREHD_ERR_INVALID, "null argument");
  if (d->in_batch) return frehd::fail(FREHD_ERR_STATE, "the domain is stepped by a batch (release it first)");
  if (!d->ready) return frehd::fail(FREHD_ERR_STATE, "domain has no state");
  OUT_TRY(cudaSetDevice(d->device));
  const int nx = d->gr.nx, pitch = d->gr.pitch;
  const long N = d->N;
  const int c = d->cur;
  const double off = d->cfg.offset;
  struct Item {
    int flag;
    const char *name;
    const double *a;
    double sub;
  };
  // DataOutput's order (fileio.c:100-121), then SubOutput's (fileio.c:145-153)
  const Item items[] = {
      {FREHD_OUT_U, "uVelocity", d->u, 0.0},         {FREHD_OUT_V, "vVelocity", d->v, 0.0},
      {FREHD_OUT_SURFACE, "surfaceZ", d->surf[c], off}, {FREHD_OUT_DEPTH, "depth", d->depth[c], 0.0},
      {FREHD_OUT_CD, "cdxp", d->CDXP, 0.0},          {FREHD_OUT_CD, "cdyp", d->CDYP, 0.0},
      {FREHD_OUT_SCALAR, "scalar", d->S[c], 0.0},    {FREHD_OUT_SUB, "SubNx", d->Nx, 0.0},
      {FREHD_OUT_SUB, "SubOy", d->Oy, 0.0},          {FREHD_OUT_SUB, "SubVx", d->Vx, 0.0},
      {FREHD_OUT_SUB, "SubVy", d->Vy, 0.0},          {FREHD_OUT_SUB, "SubV", d->V, 0.0},
      {FREHD_OUT_SUB, "SubZ", d->Z, 0.0},
  };
  frehd::FmtScratch fs;
  std::string s;
  for (const Item &it : items) {
    if (!(fields & it.flag)) continue;
    int rc = frehd::format_values(Values{it.a, nx, pitch, it.sub}, N, d->stream, fs, &s);
    if (!rc) rc = frehd::write_file(prefix, it.name, tt, s);
    if (rc) return rc;
  }
  // the tracers beside the scalar file: scalar1_<tt>.dat ...
  for (int t = 1; (fields & FREHD_OUT_SCALAR) && t < d->p.nscalar; ++t) {
    char name[16];
    std::snprintf(name, sizeof(name), "scalar%d", t);
    int rc = frehd::format_values(Values{d->Tr[t - 1][c], nx, pitch, 0.0}, N, d->stream, fs, &s);
    if (!rc) rc = frehd::write_file(prefix, name, tt, s);
    if (rc) return rc;
  }
  // DataOutput always round-trips the interior surface through the datum
  frehd::k_surf_round_trip<<<(unsigned)((N + 255) / 256), 256, 0, d->stream>>>(d->surf[c], nx,
                                                                              d->gr.ny, pitch, off);
  OUT_TRY(cudaGetLastError());
  OUT_TRY(cudaStreamSynchronize(d->stream));
  return FREHD_OK;
}

extern "C" int frehd_domain_write_restart(frehd_domain *d, const char *prefix, int tt, double tNEnd) {
  if (!d || !prefix) return frehd::fail(FREHD_ERR_INVALID, "null argument");
  if (d->in_batch) return frehd::fail(FREHD_ERR_STATE, "the domain is stepped by a batch (release it first)");
  if (!d->ready) return frehd::fail(FREHD_ERR_STATE, "domain has no state");
  OUT_TRY(cudaSetDevice(d->device));
  const int nx = d->gr.nx, pitch = d->gr.pitch;
  const long N = d->N;
  const int c = d->cur;
  const double off = d->cfg.offset;
  // [tNEnd, dx, dy, surf - offset, uu, vv, S] (fileio.c:217-238)
  std::string all, s;
  {
    std::vector<double> head = {tNEnd, d->cfg.dx, d->cfg.dy};
    int rc = frehd::host_format(head, &s);
    if (rc) return rc;
    all += s;
  }
  const Values parts[] = {{d->surf[c], nx, pitch, off}, {d->u, nx, pitch, 0.0},
                          {d->v, nx, pitch, 0.0}, {d->S[c], nx, pitch, 0.0}};
  frehd::FmtScratch fs;
  for (const Values &v : parts) {
    int rc = frehd::format_values(v, N, d->stream, fs, &s);
    if (rc) return rc;
    all += s;
  }
  int rc = frehd::write_file(prefix, "restart", tt, all);
  if (rc) return rc;
  frehd::k_surf_round_trip<<<(unsigned)((N + 255) / 256), 256, 0, d->stream>>>(d->surf[c], nx,
                                                                              d->gr.ny, pitch, off);
  OUT_TRY(cudaGetLastError());
  OUT_TRY(cudaStreamSynchronize(d->stream));
  return FREHD_OK;
}
