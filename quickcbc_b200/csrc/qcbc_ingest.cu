// Input stage of an analysis (include/qcbc_ingest.h): QuickCBC's data and PSD files read on the
// host, the data conditioned on the GPU (Tukey window, FP64 Stockham FFT, GSL half-complex
// layout, sqrt(Tobs)/N), and the PSD model of noise marginalisation evaluated on the GPU
// (natural cubic spline of the log PSD plus Lorentzian lines, Utilities.c:1908-1955).
#include <cuda_runtime.h>

#include <cctype>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/qcbc_ingest.h"
#include "qcbc_ingest_dev.h"

extern "C" int qcbc_internal_fail(int code, const char* msg);
extern "C" int qcbc_internal_ensure_init(void);

namespace qcbc {
namespace {

int ifail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return qcbc_internal_fail(code, buf);
}

#define ICU(call)                                                                             \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) return ifail(QCBC_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

// ---------------------------------------------------------------- text files
// Whole file into memory, NUL-terminated.
int slurp(const char* path, std::vector<char>& buf) {
  if (!path) return ifail(QCBC_EINVAL, "NULL path");
  FILE* f = fopen(path, "rb");
  if (!f) return ifail(QCBC_EINVAL, "cannot open %s", path);
  buf.clear();
  char chunk[1 << 16];
  size_t n;
  while ((n = fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + n);
  fclose(f);
  buf.push_back('\0');
  return QCBC_OK;
}

// Numbers of a whitespace-separated text, in the syntax fscanf("%lf") accepts (strtod's), up to
// `want` of them (want < 0: all).  *ends_in_number: the text ends right after its last number.
int parse_numbers(const char* path, const std::vector<char>& buf, long long want, std::vector<double>& out,
                  bool* ends_in_number) {
  out.clear();
  const char* p = buf.data();
  const char* end = p + buf.size() - 1;
  bool last_num = false;
  while (p < end && (want < 0 || (long long)out.size() < want)) {
    if (isspace((unsigned char)*p)) {
      ++p;
      last_num = false;
      continue;
    }
    char* e = nullptr;
    double v = strtod(p, &e);
    if (e == p) return ifail(QCBC_EINVAL, "%s: unreadable value at byte %lld", path, (long long)(p - buf.data()));
    out.push_back(v);
    p = e;
    last_num = true;
  }
  if (ends_in_number) *ends_in_number = last_num && p >= end;
  return QCBC_OK;
}

// ---------------------------------------------------------------- conditioning kernels
constexpr double kPi = 3.141592653589793238462643383279502884;

// Tukey factor of sample i (Utilities.c:635-652): cosine tapers below imin and above imax.
__device__ double tukey_factor(int i, int imin, int imax, int nwin) {
  double w = 1.0;
  if (i < imin) w = 0.5 * (1.0 + cos(kPi * ((double)i / (double)imin - 1.0)));
  if (i > imax) w = 0.5 * (1.0 + cos(kPi * ((double)(i - imax) / (double)nwin)));
  return w;
}

// Windowed real samples packed as M = N/2 complex values z[n] = x[2n] + i x[2n+1].
__global__ void k_pack_tukey(const double* __restrict__ x, int N, int imin, int imax, int nwin,
                             double2* __restrict__ z) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N / 2) return;
  z[n] = make_double2(x[2 * n] * tukey_factor(2 * n, imin, imax, nwin),
                      x[2 * n + 1] * tukey_factor(2 * n + 1, imin, imax, nwin));
}

// One radix-2 pass of the Stockham autosort FFT (Govindaraju et al., SC 2008): butterflies of
// stride M/2 with twiddles exp(-i pi k / Ns), results in natural order after log2(M) passes.
__global__ void k_fft_pass(const double2* __restrict__ in, double2* __restrict__ out, int M, int Ns) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= M / 2) return;
  const int k = j & (Ns - 1);
  double s, c;
  sincospi(-(double)k / (double)Ns, &s, &c);
  const double2 a = in[j], b0 = in[j + M / 2];
  const double2 b = make_double2(b0.x * c - b0.y * s, b0.x * s + b0.y * c);
  const int o = (j - k) * 2 + k;
  out[o] = make_double2(a.x + b.x, a.y + b.y);
  out[o + Ns] = make_double2(a.x - b.x, a.y - b.y);
}

// Spectrum of the N real samples from the M-point transform Z of the packed pairs:
// X[k] = (Z[k] + conj Z[M-k]) / 2 - i exp(-2 pi i k / N) (Z[k] - conj Z[M-k]) / 2, written in
// GSL's half-complex layout (D[k] = Re X[k], D[N-k] = Im X[k], D[0], D[N/2] real) times `scale`.
__global__ void k_unpack_real(const double2* __restrict__ Z, int N, double scale, double* __restrict__ D) {
  const int M = N / 2;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= M) return;
  if (k == 0) {
    const double2 z = Z[0];
    D[0] = (z.x + z.y) * scale;
    D[M] = (z.x - z.y) * scale;
    return;
  }
  const double2 a = Z[k], bz = Z[M - k];
  const double2 b = make_double2(bz.x, -bz.y);                 // conj Z[M-k]
  const double2 e = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
  const double2 d = make_double2(0.5 * (a.x - b.x), 0.5 * (a.y - b.y));
  const double2 o = make_double2(d.y, -d.x);                   // -i d
  double s, c;
  sincospi(-(double)k / (double)M, &s, &c);                   // exp(-2 pi i k / N)
  D[k] = (e.x + (o.x * c - o.y * s)) * scale;
  D[N - k] = (e.y + (o.x * s + o.y * c)) * scale;
}

bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// ---------------------------------------------------------------- PSD model kernels
struct ModelDev {
  const double* ffit;    // [nifo][nsp]
  const double* y;       // [nifo][nsample][nsp]
  double* c;             // [nifo][nsample][nsp] natural-spline c_i (half the second derivative)
  double* cp;            // [nifo][nsample][nsp] elimination scratch
  const double* lines;   // [nifo][nsample][nlm][5]
  int nifo, nsample, nsp, nlm;
  int nspline[3], nlines[3];
};

// One natural cubic spline per (detector, sample): h_{i-1} c_{i-1} + 2 (h_{i-1} + h_i) c_i + h_i c_{i+1}
// = 3 (dy_i / h_i - dy_{i-1} / h_{i-1}), c_0 = c_{n-1} = 0, by forward elimination and back
// substitution (the system is diagonally dominant).
__global__ void k_spline_setup(ModelDev m) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m.nifo * m.nsample) return;
  const int ifo = t / m.nsample;
  const int n = m.nspline[ifo];
  const double* x = m.ffit + (size_t)ifo * m.nsp;
  const double* y = m.y + (size_t)t * m.nsp;
  double* c = m.c + (size_t)t * m.nsp;
  double* cp = m.cp + (size_t)t * m.nsp;
  c[0] = 0.0;
  c[n - 1] = 0.0;
  double cprev = 0.0, rprev = 0.0;
  for (int i = 1; i < n - 1; i++) {
    const double hl = x[i] - x[i - 1], hr = x[i + 1] - x[i];
    const double r = 3.0 * ((y[i + 1] - y[i]) / hr - (y[i] - y[i - 1]) / hl);
    const double den = 2.0 * (hl + hr) - hl * cprev;
    cprev = hr / den;
    rprev = (r - hl * rprev) / den;
    cp[i] = cprev;
    c[i] = rprev;
  }
  for (int i = n - 3; i >= 1; i--) c[i] -= cp[i] * c[i + 1];
}

// makespec for sample k: SN[0] and SN[nh-1] from the end knots, bins 1 .. nh-2 from the spline at
// f = i / Tobs times (1 + the sum of the lines within their widths).
__global__ void k_makespec(ModelDev m, int k, int nh, double Tobs, double* __restrict__ S, int stride) {
  const int ifo = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nh) return;
  const int n = m.nspline[ifo];
  const double* x = m.ffit + (size_t)ifo * m.nsp;
  const size_t row = (size_t)ifo * m.nsample + k;
  const double* y = m.y + row * m.nsp;
  const double* c = m.c + row * m.nsp;
  double* out = S + (size_t)ifo * stride;
  if (i == 0) { out[0] = exp(y[0]); return; }
  if (i == nh - 1) { out[nh - 1] = exp(y[n - 1]); return; }
  const double f = (double)i / Tobs;
  int lo = 0, hi = n - 1;                      // largest lo with x[lo] <= f, at most n - 2
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (x[mid] > f) hi = mid; else lo = mid;
  }
  const double h = x[lo + 1] - x[lo], dy = y[lo + 1] - y[lo], dx = f - x[lo];
  const double b = dy / h - h * (c[lo + 1] + 2.0 * c[lo]) / 3.0;
  const double d = (c[lo + 1] - c[lo]) / (3.0 * h);
  const double sm = exp(y[lo] + dx * (b + dx * (c[lo] + dx * d)));
  const double* L = m.lines + row * (size_t)m.nlm * 5;
  const double ff2 = f * f;
  double sum = 0.0;
  for (int j = 0; j < m.nlines[ifo]; j++) {
    const double lf = L[5 * j], lh = L[5 * j + 1], lQ = L[5 * j + 2], lw = L[5 * j + 3], ld = L[5 * j + 4];
    const double ax = fabs(f - lf);
    if (ax < lw) {
      double z = 1.0;
      if (ax > ld) z = exp(-(ax - ld) / ld);
      const double f2 = lf * lf;
      const double df2 = lQ * (1.0 - ff2 / f2);
      sum += z * lh / (ff2 / f2 + df2 * df2);
    }
  }
  out[i] = sm * (1.0 + sum);
}

// ---------------------------------------------------------------- event weights
__global__ void k_band_min(const double* __restrict__ S, int stride, int lo, int hi, double* __restrict__ out) {
  __shared__ double red[32];
  const double* s = S + (size_t)blockIdx.x * stride;
  double m = HUGE_VAL;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const double v = s[i];
    if (v > 0.0 && v < m) m = v;
  }
  for (int o = 16; o; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : HUGE_VAL;
    for (int o = 16; o; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) out[blockIdx.x] = m;
  }
}

__global__ void k_event_weights(const double* __restrict__ D, int N, const double* __restrict__ S, int stride, int lo,
                                int hi, int nifo, Sigmas sg, double* __restrict__ w64, float* __restrict__ wm) {
  const int id = blockIdx.y;
  const int i = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= hi) return;
  const int nh = N / 2;
  const double sigma = sg.v[id];
  const double s = S[(size_t)id * stride + i];
  const double* Dr = D + (size_t)id * N;
  const double wr = 4.0 * sigma * Dr[i] / s;
  const double wi = 4.0 * sigma * Dr[N - i] / s;
  const double ws = 4.0 * sigma * sigma / s;
  double* r = w64 + (size_t)id * 3 * nh;
  r[i] = wr;
  r[nh + i] = wi;
  r[2 * nh + i] = ws;
  // the mixed kernel's planes (EventData::wm) carry the amplitude's bin factor i^{-7/6}
  const double p = pow((double)i, -7.0 / 6.0);
  const float fr = (float)(wr * p), fi = (float)(wi * p), fs = (float)(ws * (p * p));
  const size_t n = (size_t)nh;
  if (nifo == 1) {
    wm[2 * (size_t)i] = fr;
    wm[2 * (size_t)i + 1] = fi;
    wm[2 * n + i] = fs;
  } else {
    // detectors 0 and 1: (wr, wi) pairs in the first float4 plane; detector 2's pair, then the
    // ws of detectors 0 and 1, in the second plane (float4 for three detectors, float2 for two);
    // detector 2's ws in the third
    if (id < 2) {
      wm[4 * (size_t)i + 2 * id] = fr;
      wm[4 * (size_t)i + 2 * id + 1] = fi;
      if (nifo == 3) wm[4 * n + 4 * (size_t)i + 2 + id] = fs;
      else wm[4 * n + 2 * (size_t)i + id] = fs;
    } else {
      wm[4 * n + 4 * (size_t)i] = fr;
      wm[4 * n + 4 * (size_t)i + 1] = fi;
      wm[8 * n + i] = fs;
    }
  }
}

}  // namespace

void launch_band_min(const double* d_S, int stride, int nifo, int lo, int hi, double* d_out, cudaStream_t s) {
  k_band_min<<<nifo, 1024, 0, s>>>(d_S, stride, lo, hi, d_out);
}

void launch_event_weights(const double* d_D, int N, const double* d_S, int stride, int nifo, int lo, int hi,
                          Sigmas sigma, double* d_w64, float* d_wm, cudaStream_t s) {
  if (hi <= lo) return;
  dim3 grid((hi - lo + 255) / 256, nifo);
  k_event_weights<<<grid, 256, 0, s>>>(d_D, N, d_S, stride, lo, hi, nifo, sigma, d_w64, d_wm);
}

}  // namespace qcbc

using namespace qcbc;

// ---------------------------------------------------------------- PSD model
struct qcbc_psd_model {
  int device = 0;
  int nifo = 0, nsample = 0, nsp = 0, nlm = 0;
  int nspline[3] = {0, 0, 0}, nlines[3] = {0, 0, 0};
  std::vector<double> ffit;   // host copy for the range checks
  double *d_ffit = nullptr, *d_y = nullptr, *d_c = nullptr, *d_cp = nullptr, *d_lines = nullptr;
  double* d_out = nullptr;
  size_t c_out = 0;
  cudaStream_t stream = nullptr;
};

static ModelDev model_dev(const qcbc_psd_model* m) {
  ModelDev d{};
  d.ffit = m->d_ffit;
  d.y = m->d_y;
  d.c = m->d_c;
  d.cp = m->d_cp;
  d.lines = m->d_lines;
  d.nifo = m->nifo;
  d.nsample = m->nsample;
  d.nsp = m->nsp;
  d.nlm = m->nlm;
  for (int i = 0; i < 3; i++) { d.nspline[i] = m->nspline[i]; d.nlines[i] = m->nlines[i]; }
  return d;
}

static void model_free(qcbc_psd_model* m) {
  if (!m) return;
  if (m->stream) cudaStreamSynchronize(m->stream);
  cudaFree(m->d_ffit); cudaFree(m->d_y); cudaFree(m->d_c); cudaFree(m->d_cp); cudaFree(m->d_lines);
  cudaFree(m->d_out);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
}

extern "C" qcbc_psd_model* qcbc_psd_model_create(int nifo, const int* nspline, const int* nlines, int nsample,
                                                 int nspline_max, int nlines_max, const double* ffit,
                                                 const double* xspline, const double* lines) {
  if (nifo < 1 || nifo > 3 || !nspline || !nlines || nsample < 1 || nspline_max < 3 || nlines_max < 0 || !ffit ||
      !xspline || (nlines_max > 0 && !lines)) {
    ifail(QCBC_EINVAL, "bad PSD model arguments");
    return nullptr;
  }
  for (int i = 0; i < nifo; i++) {
    if (nspline[i] < 3 || nspline[i] > nspline_max || nlines[i] < 0 || nlines[i] > nlines_max) {
      ifail(QCBC_EINVAL, "detector %d: %d knots, %d lines (at least 3 knots)", i, nspline[i], nlines[i]);
      return nullptr;
    }
    for (int k = 1; k < nspline[i]; k++)
      if (!(ffit[(size_t)i * nspline_max + k] > ffit[(size_t)i * nspline_max + k - 1])) {
        ifail(QCBC_EINVAL, "detector %d: knot frequencies must increase strictly", i);
        return nullptr;
      }
  }
  if (qcbc_internal_ensure_init()) return nullptr;
  qcbc_psd_model* m = new qcbc_psd_model();
  cudaGetDevice(&m->device);
  m->nifo = nifo;
  m->nsample = nsample;
  m->nsp = nspline_max;
  m->nlm = nlines_max;
  for (int i = 0; i < nifo; i++) { m->nspline[i] = nspline[i]; m->nlines[i] = nlines[i]; }
  m->ffit.assign(ffit, ffit + (size_t)nifo * nspline_max);
  const size_t nf = (size_t)nifo * nspline_max, ny = nf * nsample,
               nl = (size_t)nifo * nsample * std::max(nlines_max, 1) * 5;
  bool ok = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&m->d_ffit, nf * 8) == cudaSuccess && cudaMalloc(&m->d_y, ny * 8) == cudaSuccess &&
            cudaMalloc(&m->d_c, ny * 8) == cudaSuccess && cudaMalloc(&m->d_cp, ny * 8) == cudaSuccess &&
            cudaMalloc(&m->d_lines, nl * 8) == cudaSuccess;
  if (!ok) {
    model_free(m);
    ifail(QCBC_ENOMEM, "PSD model of %d samples", nsample);
    return nullptr;
  }
  ok = cudaMemcpy(m->d_ffit, ffit, nf * 8, cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemcpy(m->d_y, xspline, ny * 8, cudaMemcpyHostToDevice) == cudaSuccess &&
       (nlines_max == 0 ||
        cudaMemcpy(m->d_lines, lines, (size_t)nifo * nsample * nlines_max * 5 * 8, cudaMemcpyHostToDevice) ==
            cudaSuccess);
  if (ok) {
    const int T = nifo * nsample;
    k_spline_setup<<<(T + 127) / 128, 128, 0, m->stream>>>(model_dev(m));
    ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(m->stream) == cudaSuccess;
  }
  if (!ok) {
    model_free(m);
    ifail(QCBC_ECUDA, "PSD model upload or spline setup failed");
    return nullptr;
  }
  return m;
}

extern "C" int qcbc_psd_model_info(const qcbc_psd_model* m, int* nifo, int* nsample, int* nspline_max,
                                   int* nlines_max) {
  if (!m) return ifail(QCBC_EINVAL, "NULL model");
  if (nifo) *nifo = m->nifo;
  if (nsample) *nsample = m->nsample;
  if (nspline_max) *nspline_max = m->nsp;
  if (nlines_max) *nlines_max = m->nlm;
  return QCBC_OK;
}

extern "C" int qcbc_psd_model_close(qcbc_psd_model* m) {
  model_free(m);
  return QCBC_OK;
}

namespace qcbc {

int psd_model_nifo(const qcbc_psd_model* m) { return m ? m->nifo : 0; }

int psd_model_draw_dev(qcbc_psd_model* m, int k, double Tobs, int N, double* d_S, int stride, cudaStream_t s) {
  if (!m || !d_S) return ifail(QCBC_EINVAL, "NULL argument");
  if (k < 0 || k >= m->nsample) return ifail(QCBC_EINVAL, "sample %d of %d", k, m->nsample);
  if (N < 8 || (N & 1) || !(Tobs > 0.0) || stride < N / 2) return ifail(QCBC_EINVAL, "bad N, Tobs or stride");
  const int nh = N / 2;
  // the spline is evaluated at 1/Tobs .. (nh-2)/Tobs; the reference's GSL spline has no
  // extrapolation (its error handler aborts), so a bin outside the knots is an error here
  const double flo = 1.0 / Tobs, fhi = (double)(nh - 2) / Tobs;
  for (int i = 0; i < m->nifo; i++) {
    const double* x = &m->ffit[(size_t)i * m->nsp];
    if (nh > 2 && (flo < x[0] || fhi > x[m->nspline[i] - 1]))
      return ifail(QCBC_EDOM, "detector %d: bins %g..%g Hz outside the knots %g..%g Hz", i, flo, fhi, x[0],
                   x[m->nspline[i] - 1]);
  }
  dim3 grid((nh + 255) / 256, m->nifo);
  k_makespec<<<grid, 256, 0, s>>>(model_dev(m), k, nh, Tobs, d_S, stride);
  ICU(cudaGetLastError());
  return QCBC_OK;
}

}  // namespace qcbc

extern "C" int qcbc_psd_draw(qcbc_psd_model* m, int k, double Tobs, int N, double* SN, int sn_stride) {
  if (!m || !SN) return ifail(QCBC_EINVAL, "NULL argument");
  if (sn_stride < N / 2) return ifail(QCBC_EINVAL, "sn_stride < N/2");
  const int nh = N / 2;
  const size_t need = (size_t)m->nifo * nh;
  if (need > m->c_out) {
    cudaFree(m->d_out);
    m->d_out = nullptr;
    m->c_out = 0;
    ICU(cudaMalloc(&m->d_out, need * 8));
    m->c_out = need;
  }
  int rc = psd_model_draw_dev(m, k, Tobs, N, m->d_out, nh, m->stream);
  if (rc) return rc;
  for (int i = 0; i < m->nifo; i++)
    ICU(cudaMemcpyAsync(SN + (size_t)i * sn_stride, m->d_out + (size_t)i * nh, (size_t)nh * 8,
                        cudaMemcpyDeviceToHost, m->stream));
  ICU(cudaStreamSynchronize(m->stream));
  return QCBC_OK;
}

extern "C" void qcbc_gpu_makespec(int Nspline, int Nlines, double* ffit, double* Sspline, double* linef, double* lineh,
                                  double* lineQ, double* linew, double* deltafmax, double* SN, double Tobs, int N) {
  std::vector<double> L((size_t)std::max(Nlines, 0) * 5);
  for (int j = 0; j < Nlines; j++) {
    L[5 * j] = linef[j];
    L[5 * j + 1] = lineh[j];
    L[5 * j + 2] = lineQ[j];
    L[5 * j + 3] = linew[j];
    L[5 * j + 4] = deltafmax[j];
  }
  const int ns[1] = {Nspline}, nl[1] = {std::max(Nlines, 0)};
  qcbc_psd_model* m = qcbc_psd_model_create(1, ns, nl, 1, Nspline, std::max(Nlines, 0), ffit, Sspline, L.data());
  if (!m) return;   // the reason is in qcbc_last_error(); SN is left as it was
  qcbc_psd_draw(m, 0, Tobs, N, SN, N / 2);
  qcbc_psd_model_close(m);
}

extern "C" void makespec(int Nspline, int Nlines, double* ffit, double* Sspline, double* linef, double* lineh,
                         double* lineQ, double* linew, double* deltafmax, double* SN, double Tobs, int N) {
  qcbc_gpu_makespec(Nspline, Nlines, ffit, Sspline, linef, lineh, lineQ, linew, deltafmax, SN, Tobs, N);
}

// ---------------------------------------------------------------- files
extern "C" int qcbc_framed_length(const char* path, int* N) {
  if (!N) return ifail(QCBC_EINVAL, "NULL argument");
  std::vector<char> buf;
  std::vector<double> v;
  bool tail = false;
  int rc = slurp(path, buf);
  if (rc == QCBC_OK) rc = parse_numbers(path, buf, -1, v, &tail);
  if (rc) return rc;
  if (v.size() % 2) return ifail(QCBC_EINVAL, "%s: %zu values, not whole rows of two", path, v.size());
  long long n = (long long)(v.size() / 2) - (tail ? 1 : 0);
  if (n > (1LL << 30)) return ifail(QCBC_EINVAL, "%s: too many rows", path);
  *N = (int)std::max(n, 0LL);
  return QCBC_OK;
}

static int read_columns(const char* path, int rows, int ncol, double* a, int ca, double* b, int cb) {
  if (rows < 0) return ifail(QCBC_EINVAL, "negative row count");
  std::vector<char> buf;
  std::vector<double> v;
  int rc = slurp(path, buf);
  if (rc == QCBC_OK) rc = parse_numbers(path, buf, (long long)rows * ncol, v, nullptr);
  if (rc) return rc;
  if ((long long)v.size() < (long long)rows * ncol)
    return ifail(QCBC_EINVAL, "%s: %zu values, %lld needed", path, v.size(), (long long)rows * ncol);
  for (int i = 0; i < rows; i++) {
    if (a) a[i] = v[(size_t)i * ncol + ca];
    if (b) b[i] = v[(size_t)i * ncol + cb];
  }
  return QCBC_OK;
}

extern "C" int qcbc_read_framed(const char* path, int N, double* t, double* x) {
  if (!x) return ifail(QCBC_EINVAL, "NULL argument");
  return read_columns(path, N, 2, t, 0, x, 1);
}

extern "C" int qcbc_read_spec(const char* path, int nh, double* SN, double* SM) {
  if (!SN) return ifail(QCBC_EINVAL, "NULL argument");
  return read_columns(path, nh, 4, SN, 1, SM, 2);
}

extern "C" int qcbc_analysis_paths(const char* dir, double Tobs, double ttrig, int label, char* framed, char* spec,
                                   int cap) {
  if (!dir || cap <= 0) return ifail(QCBC_EINVAL, "NULL directory or no room");
  const char* sep = (dir[0] && dir[strlen(dir) - 1] != '/') ? "/" : "";
  int a = 0, b = 0;
  if (framed) a = snprintf(framed, (size_t)cap, "%s%sframed_%d_%d_%d.dat", dir, sep, (int)Tobs, (int)ttrig, label);
  if (spec) b = snprintf(spec, (size_t)cap, "%s%sspec_%d_%d_%d.dat", dir, sep, (int)Tobs, (int)ttrig, label);
  if (a >= cap || b >= cap) return ifail(QCBC_EINVAL, "path longer than %d bytes", cap);
  return QCBC_OK;
}

// ---------------------------------------------------------------- conditioning
extern "C" int qcbc_condition_data(int nifo, int N, double Tobs, const double* x, int x_stride, double* D,
                                   int d_stride) {
  if (nifo < 1 || !x || !D) return ifail(QCBC_EINVAL, "NULL argument or no detectors");
  if (N < 8 || !pow2(N)) return ifail(QCBC_EINVAL, "N=%d: the radix-2 transform needs a power of two >= 8", N);
  if (!(Tobs > 0.0) || x_stride < N || d_stride < N) return ifail(QCBC_EINVAL, "bad Tobs or strides");
  int rc = qcbc_internal_ensure_init();
  if (rc) return rc;
  // Tukey window with a 0.4 s rise (QuickCBC.c:244-246; Utilities.c:635-652)
  const double alpha = 2.0 * 0.4 / Tobs;
  const int imin = (int)(alpha * (double)(N - 1) / 2.0);
  const int imax = (int)((double)(N - 1) * (1.0 - alpha / 2.0));
  const int nwin = N - imax;
  const int M = N / 2;
  const double scale = sqrt(Tobs) / (double)N;        // QuickCBC.c:309-313
  double* d_x = nullptr;
  double* d_D = nullptr;
  double2 *d_a = nullptr, *d_b = nullptr;
  cudaStream_t s = nullptr;
  auto cleanup = [&]() {
    if (s) cudaStreamSynchronize(s);
    cudaFree(d_x); cudaFree(d_D); cudaFree(d_a); cudaFree(d_b);
    if (s) cudaStreamDestroy(s);
  };
  bool ok = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&d_x, (size_t)N * 8) == cudaSuccess && cudaMalloc(&d_D, (size_t)N * 8) == cudaSuccess &&
            cudaMalloc(&d_a, (size_t)M * 16) == cudaSuccess && cudaMalloc(&d_b, (size_t)M * 16) == cudaSuccess;
  if (!ok) { cleanup(); return ifail(QCBC_ENOMEM, "conditioning buffers for N=%d", N); }
  for (int id = 0; id < nifo && ok; id++) {
    ok = cudaMemcpyAsync(d_x, x + (size_t)id * x_stride, (size_t)N * 8, cudaMemcpyHostToDevice, s) == cudaSuccess;
    k_pack_tukey<<<(M + 255) / 256, 256, 0, s>>>(d_x, N, imin, imax, nwin, d_a);
    double2 *in = d_a, *out = d_b;
    for (int Ns = 1; Ns < M; Ns *= 2) {
      k_fft_pass<<<(M / 2 + 255) / 256, 256, 0, s>>>(in, out, M, Ns);
      std::swap(in, out);
    }
    k_unpack_real<<<(M + 255) / 256, 256, 0, s>>>(in, N, scale, d_D);
    ok = ok && cudaGetLastError() == cudaSuccess &&
         cudaMemcpyAsync(D + (size_t)id * d_stride, d_D, (size_t)N * 8, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
         cudaStreamSynchronize(s) == cudaSuccess;
  }
  cleanup();
  return ok ? QCBC_OK : ifail(QCBC_ECUDA, "conditioning failed: %s", cudaGetErrorString(cudaGetLastError()));
}

extern "C" int qcbc_load_analysis(const char* dir, double Tobs, double ttrig, int nifo, const int* labels, int N,
                                  double* D, int d_stride, double* SN, double* SM, int sn_stride) {
  if (!dir || !labels || !D || !SN || nifo < 1 || nifo > 3) return ifail(QCBC_EINVAL, "bad arguments");
  if (d_stride < N || sn_stride < N / 2) return ifail(QCBC_EINVAL, "row strides too small");
  std::vector<double> x((size_t)nifo * N);
  char fr[4096], sp[4096];
  for (int id = 0; id < nifo; id++) {
    int rc = qcbc_analysis_paths(dir, Tobs, ttrig, labels[id], fr, sp, (int)sizeof(fr));
    if (rc == QCBC_OK) rc = qcbc_read_framed(fr, N, nullptr, &x[(size_t)id * N]);
    if (rc == QCBC_OK)
      rc = qcbc_read_spec(sp, N / 2, SN + (size_t)id * sn_stride, SM ? SM + (size_t)id * sn_stride : nullptr);
    if (rc) return rc;
  }
  return qcbc_condition_data(nifo, N, Tobs, x.data(), N, D, d_stride);
}

// PSD sample files (QuickCBC.c:322-378).  Nsample is the last detector's summary value, as there.
extern "C" qcbc_psd_model* qcbc_psd_model_open(const char* dir, int nifo, const int* labels) {
  if (!dir || !labels || nifo < 1 || nifo > 3) { ifail(QCBC_EINVAL, "bad arguments"); return nullptr; }
  const char* sep = (dir[0] && dir[strlen(dir) - 1] != '/') ? "/" : "";
  char path[4096];
  int nsp[3] = {0, 0, 0}, nln[3] = {0, 0, 0}, nsample = 0, nspm = 0, nlm = 0;
  std::vector<char> buf;
  std::vector<double> v;
  for (int j = 0; j < nifo; j++) {
    snprintf(path, sizeof(path), "%s%ssummary_%d.dat", dir, sep, labels[j]);
    if (slurp(path, buf) || parse_numbers(path, buf, 3, v, nullptr)) return nullptr;
    if (v.size() < 3) { ifail(QCBC_EINVAL, "%s: three counts expected", path); return nullptr; }
    nsp[j] = (int)v[0];
    nln[j] = (int)v[1];
    nsample = (int)v[2];
    nspm = std::max(nspm, nsp[j]);
    nlm = std::max(nlm, nln[j]);
  }
  if (nsample < 1 || nspm < 3 || nlm < 0) { ifail(QCBC_EINVAL, "summary: bad counts"); return nullptr; }
  std::vector<double> ffit((size_t)nifo * nspm, 0.0), xs((size_t)nifo * nsample * nspm, 0.0),
      lines((size_t)nifo * nsample * std::max(nlm, 1) * 5, 0.0);
  for (int j = 0; j < nifo; j++) {
    snprintf(path, sizeof(path), "%s%ssfile_%d.dat", dir, sep, labels[j]);
    if (slurp(path, buf) || parse_numbers(path, buf, (long long)nsample * nsp[j], v, nullptr)) return nullptr;
    if ((long long)v.size() < (long long)nsample * nsp[j]) { ifail(QCBC_EINVAL, "%s: short", path); return nullptr; }
    for (int i = 0; i < nsample; i++)
      for (int k = 0; k < nsp[j]; k++) xs[((size_t)j * nsample + i) * nspm + k] = v[(size_t)i * nsp[j] + k];
    snprintf(path, sizeof(path), "%s%sffile_%d.dat", dir, sep, labels[j]);
    if (slurp(path, buf) || parse_numbers(path, buf, nsp[j], v, nullptr)) return nullptr;
    if ((int)v.size() < nsp[j]) { ifail(QCBC_EINVAL, "%s: short", path); return nullptr; }
    for (int k = 0; k < nsp[j]; k++) ffit[(size_t)j * nspm + k] = v[k];
    snprintf(path, sizeof(path), "%s%slfile_%d.dat", dir, sep, labels[j]);
    const long long nv = (long long)nsample * nln[j] * 5;
    if (nln[j] > 0) {
      if (slurp(path, buf) || parse_numbers(path, buf, nv, v, nullptr)) return nullptr;
      if ((long long)v.size() < nv) { ifail(QCBC_EINVAL, "%s: short", path); return nullptr; }
      for (int i = 0; i < nsample; i++)
        for (int k = 0; k < nln[j]; k++)
          for (int q = 0; q < 5; q++)
            lines[(((size_t)j * nsample + i) * nlm + k) * 5 + q] = v[((size_t)i * nln[j] + k) * 5 + q];
    }
  }
  return qcbc_psd_model_create(nifo, nsp, nln, nsample, nspm, nlm, ffit.data(), xs.data(), lines.data());
}
