// C ABI of libfd3: plan setup (host), workspace layout and the stream-ordered pipelines.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <new>

#include "fd3_internal.h"

using namespace fd3;

struct fd3_plan {
  int S = 0, R = 0, method = 0, P = 0, precision = 0;
  int edge_cutoff = 0;   // 1: edge-list edges at or beyond the CN cutoff contribute nothing
  MeshGeom mg{};
  int ens[3] = {0, 0, 0};
  Tables h_tab{};
  Tables* d_tab = nullptr;
  double* d_eigvecs = nullptr;
  GreenPair* d_green = nullptr;
  GreenPairF* d_green_f = nullptr;
  // D4 k-space CN: pair constants, self terms, (S channels) 3D transforms
  int cnfunc = FD3_CN_SMOOTH;
  CnPair* d_cnpair = nullptr;
  double* d_cnself = nullptr;
  cufftHandle fwd_cn = 0, inv_cn = 0;
  float* d_deconv = nullptr;
  float* d_win_axes = nullptr;
  cufftHandle fwd = 0, inv = 0;
  bool has_fft = false;
  cufftHandle fwd2 = 0, inv2 = 0;   // (y, z) 2D transforms of the fused x-pass path
  bool has_fft2 = false;
  size_t fft_ws = 0;
  // side stream of the fused entry: the mesh sort (positions only) runs beside the cell list and
  // the CN stage, forked from and joined back to the caller's stream by events (also under capture)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // optional per-stage CUDA-event timing (fd3_profile_enable / fd3_profile_read)
  static constexpr int kMaxMarks = 24;
  bool prof = false;
  cudaEvent_t ev[kMaxMarks] = {};
  const char* mark_name[kMaxMarks] = {};
  int n_marks = 0;
};

// Record a stage boundary on the launching stream when profiling is on.
static void prof_begin(fd3_plan* p, cudaStream_t s) {
  p->n_marks = 0;
  if (!p->prof) return;
  cudaEventRecord(p->ev[0], s);
  p->mark_name[0] = "start";
  p->n_marks = 1;
}
static void prof_mark(fd3_plan* p, cudaStream_t s, const char* name) {
  if (!p->prof || p->n_marks >= fd3_plan::kMaxMarks) return;
  cudaEventRecord(p->ev[p->n_marks], s);
  p->mark_name[p->n_marks++] = name;
}

// ------------------------------------------------------------------ errors / counters
namespace fd3 {
static thread_local char g_err[512] = "";
void set_error(const char* where, const char* what) { snprintf(g_err, sizeof(g_err), "%s: %s", where, what); }
static std::atomic<int64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
}  // namespace fd3

extern "C" const char* fd3_last_error(void) { return g_err; }
extern "C" int64_t fd3_launch_count(void) { return g_launches.load(); }

#define FD3_CUFFT(call)                                       \
  do {                                                        \
    cufftResult r_ = (call);                                  \
    if (r_ != CUFFT_SUCCESS) {                                \
      char b_[64];                                            \
      snprintf(b_, sizeof(b_), "cufft status %d", (int)r_);   \
      set_error(#call, b_);                                   \
      return FD3_ECUFFT;                                      \
    }                                                         \
  } while (0)
#define FD3_TRY(x)          \
  do {                      \
    int rc_ = (x);          \
    if (rc_) return rc_;    \
  } while (0)

// ------------------------------------------------------------------ plan
static int largest_divisor_le(int n, int cap) {
  for (int t = cap; t >= 1; --t)
    if (n % t == 0) return t;
  return 1;
}

extern "C" int fd3_plan_create(const fd3_plan_desc* d, fd3_plan** out) {
  if (!d || !out) return FD3_EINVAL;
  *out = nullptr;
  const int S = d->n_species, R = d->n_rank;
  if (S < 1 || S > FD3_MAX_SPECIES || R < 1 || R > FD3_MAX_RANK) {
    set_error("fd3_plan_create", "n_species must be 1..64 and n_rank 1..32");
    return FD3_EINVAL;
  }
  if (d->method != FD3_METHOD_SPME && d->method != FD3_METHOD_PME && d->method != FD3_METHOD_EWALD) return FD3_EINVAL;
  if (d->precision != FD3_PREC_FP64 && d->precision != FD3_PREC_MIXED) return FD3_EINVAL;
  if (d->cnfunc != FD3_CN_SMOOTH && d->cnfunc != FD3_CN_D4) {
    set_error("fd3_plan_create", "cnfunc must be FD3_CN_SMOOTH or FD3_CN_D4");
    return FD3_EINVAL;
  }
  if (d->cnfunc == FD3_CN_D4) {
    if (d->method == FD3_METHOD_EWALD || S > kCn4MaxSpecies || !d->rcov_cn || !d->en) {
      set_error("fd3_plan_create", "the D4 k-space CN needs method spme or pme, at most 8 species, rcov_cn and en");
      return FD3_EINVAL;
    }
  }
  const bool mesh = d->method != FD3_METHOD_EWALD;
  if (mesh) {
    if (d->order < 1 || d->order > FD3_MAX_ORDER) {
      set_error("fd3_plan_create", "interpolation order must be 1..8");
      return FD3_EINVAL;
    }
    for (int a = 0; a < 3; ++a)
      if (d->mesh[a] < 1) return FD3_EINVAL;
  }
  if (!mesh) {
    for (int a = 0; a < 3; ++a)
      if (d->ewald_ns[a] < 1) {
        set_error("fd3_plan_create", "ewald_ns must be >= 1 on every axis");
        return FD3_EINVAL;
      }
    if ((int64_t)d->ewald_ns[0] * d->ewald_ns[1] * d->ewald_ns[2] > (int64_t)1 << 28) {
      set_error("fd3_plan_create", "ewald k-vector box too large");
      return FD3_EINVAL;
    }
  }
  fd3_plan* p = new (std::nothrow) fd3_plan();
  if (!p) return FD3_EINVAL;
  p->S = S;
  p->R = R;
  p->method = d->method;
  p->P = d->order;
  p->precision = d->precision;
  for (int a = 0; a < 3; ++a) p->ens[a] = d->ewald_ns[a];

  Tables& t = p->h_tab;
  memset(&t, 0, sizeof(t));
  t.n_species = S;
  t.n_rank = R;
  t.s6 = d->params[0];
  t.s8 = d->params[1];
  t.r_cut = d->r_cut;
  // cncorr belongs to the smooth-cutoff CN (core.py:383-384); the D4 CN does not apply it
  t.has_cncorr = d->has_cncorr && d->cncorr && d->cnfunc == FD3_CN_SMOOTH;
  p->cnfunc = d->cnfunc;
  for (int s = 0; s < S; ++s) {
    t.rcov[s] = d->rcov[s];
    for (int q = 0; q < 7; ++q) t.cnref[7 * s + q] = d->cnref[7 * s + q];
    if (t.has_cncorr) {
      t.cncorr[2 * s] = d->cncorr[2 * s];
      t.cncorr[2 * s + 1] = d->cncorr[2 * s + 1];
    }
  }
  for (int r = 0; r < R; ++r) t.eigs[r] = d->eigs[r];
  // Green's function constants per species pair (pair_pot.py:55-105) and phi_XX(0) (:84-89)
  GreenPair* gp = new GreenPair[S * S];
  const double pi = kPi, pi2 = pi * pi;
  const double a1 = d->params[2], a2 = d->params[3];
  for (int X = 0; X < S; ++X)
    for (int Y = 0; Y < S; ++Y) {
      GreenPair& g = gp[X * S + Y];
      g.qq = d->sqrtq[X] * d->sqrtq[Y];
      g.R = a1 * sqrt(3.0 * g.qq) + a2;
      const double R2 = g.R * g.R, R3 = R2 * g.R, R4 = g.R * R3, R5 = g.R * R4, R6 = R3 * R3;
      g.c6s1 = (2.0 * pi2) / (3.0 * R3);
      g.c6s2 = (2.0 * pi2 * g.R) / 9.0;
      g.c6pre = (2.0 * pi2) / (3.0 * R4);
      g.c8s1 = (pi2 * sqrt(2.0) * sin(pi / 8.0)) / R5;
      g.c8s2 = g.c8s1 * R2 / 6.0;
      g.c8pre = -pi2 / R6;
      if (X == Y) {
        const double R8 = R3 * R5;
        t.selfcont[X] = t.s6 / R6 + 3.0 * t.s8 * g.qq / R8;
      }
    }
  GreenPairF* gpf = new GreenPairF[S * S];
  for (int k = 0; k < S * S; ++k)
    gpf[k] = GreenPairF{(float)gp[k].R, (float)gp[k].qq, (float)gp[k].c6s1, (float)gp[k].c6s2, (float)gp[k].c6pre,
                        (float)gp[k].c8s1, (float)gp[k].c8s2, (float)gp[k].c8pre};
  int rc = FD3_OK;
  do {
    if (cudaMalloc(&p->d_tab, sizeof(Tables)) != cudaSuccess ||
        cudaMalloc(&p->d_eigvecs, sizeof(double) * S * 7 * R) != cudaSuccess ||
        cudaMalloc(&p->d_green, sizeof(GreenPair) * S * S) != cudaSuccess ||
        cudaMalloc(&p->d_green_f, sizeof(GreenPairF) * S * S) != cudaSuccess) {
      set_error("fd3_plan_create", "cudaMalloc of the species tables failed");
      rc = FD3_ECUDA;
      break;
    }
    if (cudaMemcpy(p->d_tab, &t, sizeof(Tables), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(p->d_eigvecs, d->eigvecs, sizeof(double) * S * 7 * R, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(p->d_green, gp, sizeof(GreenPair) * S * S, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(p->d_green_f, gpf, sizeof(GreenPairF) * S * S, cudaMemcpyHostToDevice) != cudaSuccess) {
      set_error("fd3_plan_create", "upload of the species tables failed");
      rc = FD3_ECUDA;
      break;
    }
    if (mesh) {
      MeshGeom& m = p->mg;
      for (int a = 0; a < 3; ++a) {
        m.n[a] = d->mesh[a];
        m.t[a] = largest_divisor_le(m.n[a], a == 2 ? 8 : 16);   // spread tile 16 x 16 x 8
        m.nt[a] = m.n[a] / m.t[a];
        const int need = 1 + (d->order - 1 + m.t[a] - 1) / m.t[a];
        m.ns[a] = need < m.nt[a] ? need : m.nt[a];
      }
      m.nzh = m.n[2] / 2 + 1;
      m.order = d->order;
      m.lagrange = d->method == FD3_METHOD_PME;
      m.S = S;
      m.R = R;
      m.filter_kt = -1;
      m.spread_zc = -1;
      m.spread_cap = 0;
      m.xpencil = -1;
      m.xq = -1;
      m.xranks = -1;
      m.filter_mma = -1;
      m.gather_tile = -1;
      m.fft_yz = -1;
      m.qpitch = 0;
      m.fft_x = -1;   // default: off (3D cuFFT around the separate filter measured faster on B200)
      const size_t Mh = (size_t)m.n[0] * m.n[1] * m.nzh;
      m.win_axes = nullptr;
      if (d->method == FD3_METHOD_SPME && d->precision == FD3_PREC_MIXED) {
        // sinc(m/n)^(2p) per axis (fftfreq order on x and y, rfftfreq on z), float64 rounded to float
        const int na = m.n[0] + m.n[1] + m.nzh;
        float* hw = new float[na];
        for (int a = 0, o = 0; a < 3; ++a) {
          const int cnt = a < 2 ? m.n[a] : m.nzh;
          for (int i = 0; i < cnt; ++i) {
            const int mm = (a < 2 && i > (m.n[a] - 1) / 2) ? i - m.n[a] : i;
            const double x = (double)mm / m.n[a];
            const double sc = x == 0.0 ? 1.0 : sin(kPi * x) / (kPi * x);
            hw[o + i] = (float)pow(sc, 2.0 * d->order);
          }
          o += cnt;
        }
        const bool ok = cudaMalloc(&p->d_win_axes, sizeof(float) * na) == cudaSuccess &&
                        cudaMemcpy(p->d_win_axes, hw, sizeof(float) * na, cudaMemcpyHostToDevice) == cudaSuccess;
        delete[] hw;
        if (!ok) {
          set_error("fd3_plan_create", "upload of the per-axis window failed");
          rc = FD3_ECUDA;
          break;
        }
        m.win_axes = p->d_win_axes;
      }
      if (d->method == FD3_METHOD_SPME && d->deconv) {
        if (cudaMalloc(&p->d_deconv, sizeof(float) * Mh) != cudaSuccess ||
            cudaMemcpy(p->d_deconv, d->deconv, sizeof(float) * Mh, cudaMemcpyHostToDevice) != cudaSuccess) {
          set_error("fd3_plan_create", "upload of the deconvolution window failed");
          rc = FD3_ECUDA;
          break;
        }
      }
      // batched 3D real transforms over the S*R channels (only library call of the pipeline)
      // 64-bit plan: C * M passes 2^31 elements for many-species boxes on 256^3 meshes
      long long n[3] = {m.n[0], m.n[1], m.n[2]};
      const long long C = (long long)S * R;
      const long long M = (long long)m.n[0] * m.n[1] * m.n[2];
      const long long Mhi = (long long)Mh;
      const bool dp = d->precision == FD3_PREC_FP64;
      size_t ws1 = 0, ws2 = 0;
      cufftResult fr;
      if ((fr = cufftCreate(&p->fwd)) != CUFFT_SUCCESS || (fr = cufftCreate(&p->inv)) != CUFFT_SUCCESS ||
          (fr = cufftSetAutoAllocation(p->fwd, 0)) != CUFFT_SUCCESS ||
          (fr = cufftSetAutoAllocation(p->inv, 0)) != CUFFT_SUCCESS ||
          (fr = cufftMakePlanMany64(p->fwd, 3, n, nullptr, 1, M, nullptr, 1, Mhi, dp ? CUFFT_D2Z : CUFFT_R2C, C,
                                    &ws1)) != CUFFT_SUCCESS ||
          (fr = cufftMakePlanMany64(p->inv, 3, n, nullptr, 1, Mhi, nullptr, 1, M, dp ? CUFFT_Z2D : CUFFT_C2R, C,
                                    &ws2)) != CUFFT_SUCCESS) {
        char b[64];
        snprintf(b, sizeof(b), "cufft status %d", (int)fr);
        set_error("fd3_plan_create: cufft plan", b);
        rc = FD3_ECUFFT;
        break;
      }
      p->has_fft = true;
      p->fft_ws = ws1 > ws2 ? ws1 : ws2;
      // (y, z) planes for the fused x-pass: batch over the C channels and nx planes
      if (xfilter_pencil(m, dp ? 1 : 0) > 0 || (!dp && xpass_applies(m, 8, 1))) {
        long long n2d[2] = {m.n[1], m.n[2]};
        const long long pr = (long long)m.n[1] * m.n[2], pc = (long long)m.n[1] * m.nzh;
        size_t ws3 = 0, ws4 = 0;
        if ((fr = cufftCreate(&p->fwd2)) != CUFFT_SUCCESS || (fr = cufftCreate(&p->inv2)) != CUFFT_SUCCESS ||
            (fr = cufftSetAutoAllocation(p->fwd2, 0)) != CUFFT_SUCCESS ||
            (fr = cufftSetAutoAllocation(p->inv2, 0)) != CUFFT_SUCCESS ||
            (fr = cufftMakePlanMany64(p->fwd2, 2, n2d, nullptr, 1, pr, nullptr, 1, pc, dp ? CUFFT_D2Z : CUFFT_R2C,
                                      C * m.n[0], &ws3)) != CUFFT_SUCCESS ||
            (fr = cufftMakePlanMany64(p->inv2, 2, n2d, nullptr, 1, pc, nullptr, 1, pr, dp ? CUFFT_Z2D : CUFFT_C2R,
                                      C * m.n[0], &ws4)) != CUFFT_SUCCESS) {
          char b[64];
          snprintf(b, sizeof(b), "cufft status %d", (int)fr);
          set_error("fd3_plan_create: cufft 2D plan", b);
          rc = FD3_ECUFFT;
          break;
        }
        p->has_fft2 = true;
        if (ws3 > p->fft_ws) p->fft_ws = ws3;
        if (ws4 > p->fft_ws) p->fft_ws = ws4;
      }
      if (d->cnfunc == FD3_CN_D4) {
        // D4 CN: 3D transforms of the S species channels, the erfc pair constants and self terms
        size_t ws5 = 0, ws6 = 0;
        if ((fr = cufftCreate(&p->fwd_cn)) != CUFFT_SUCCESS || (fr = cufftCreate(&p->inv_cn)) != CUFFT_SUCCESS ||
            (fr = cufftSetAutoAllocation(p->fwd_cn, 0)) != CUFFT_SUCCESS ||
            (fr = cufftSetAutoAllocation(p->inv_cn, 0)) != CUFFT_SUCCESS ||
            (fr = cufftMakePlanMany64(p->fwd_cn, 3, n, nullptr, 1, M, nullptr, 1, Mhi, dp ? CUFFT_D2Z : CUFFT_R2C,
                                      S, &ws5)) != CUFFT_SUCCESS ||
            (fr = cufftMakePlanMany64(p->inv_cn, 3, n, nullptr, 1, Mhi, nullptr, 1, M, dp ? CUFFT_Z2D : CUFFT_C2R,
                                      S, &ws6)) != CUFFT_SUCCESS) {
          char b[64];
          snprintf(b, sizeof(b), "cufft status %d", (int)fr);
          set_error("fd3_plan_create: cufft CN plan", b);
          rc = FD3_ECUFFT;
          break;
        }
        if (ws5 > p->fft_ws) p->fft_ws = ws5;
        if (ws6 > p->fft_ws) p->fft_ws = ws6;
        CnPair* cp = new CnPair[S * S];
        double* cs = new double[S];
        const double A = 1.0 / 3.0 + 1.0 / (2.0 * kCn4K0 * kCn4K0);                   // pair_pot.py:321-324
        const double B = 1.0 / 30.0 + 1.0 / (6.0 * kCn4K0 * kCn4K0) + 1.0 / (8.0 * pow(kCn4K0, 4.0));
        for (int X = 0; X < S; ++X)
          for (int Y = 0; Y < S; ++Y) {
            CnPair& c = cp[X * S + Y];
            c.r0 = d->rcov_cn[X] + d->rcov_cn[Y];
            const double ed = fabs(d->en[X] - d->en[Y]) + kCn4K2;
            c.delta = kCn4K1 * exp(-ed * ed / kCn4K3);
            c.c0 = 4.0 * kPi * c.delta * c.r0 * c.r0 * c.r0 * A;
            c.c2 = 4.0 * kPi * c.delta * c.r0 * c.r0 * c.r0 * c.r0 * c.r0 * B;
            if (X == Y) cs[X] = c.delta / 2.0 * erfc(-kCn4K0);                        // pair_pot.py:330-331
          }
        const bool ok = cudaMalloc(&p->d_cnpair, sizeof(CnPair) * S * S) == cudaSuccess &&
                        cudaMalloc(&p->d_cnself, sizeof(double) * S) == cudaSuccess &&
                        cudaMemcpy(p->d_cnpair, cp, sizeof(CnPair) * S * S, cudaMemcpyHostToDevice) == cudaSuccess &&
                        cudaMemcpy(p->d_cnself, cs, sizeof(double) * S, cudaMemcpyHostToDevice) == cudaSuccess;
        delete[] cp;
        delete[] cs;
        if (!ok) {
          set_error("fd3_plan_create", "upload of the D4 CN constants failed");
          rc = FD3_ECUDA;
          break;
        }
      }
      // side stream and fork/join events of the fused entry (without them it runs on one stream)
      if (cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (p->ev_fork) cudaEventDestroy(p->ev_fork);
        if (p->side) cudaStreamDestroy(p->side);
        p->side = nullptr;
        p->ev_fork = p->ev_join = nullptr;
      }
    }
  } while (0);
  delete[] gp;
  delete[] gpf;
  if (rc) {
    fd3_plan_destroy(p);
    return rc;
  }
  *out = p;
  return FD3_OK;
}

// Unit shape of the TMA x-pass in effect: q values per unit (default 16: one 128-byte line per
// spectrum row) and ranks per unit (default 1).
static void xpass_shape(const fd3_plan* p, int* Q, int* RG) {
  *Q = p->mg.xq > 0 ? p->mg.xq : 16;
  *RG = p->mg.xranks > 0 ? p->mg.xranks : 1;
}
static bool xpass_on(const fd3_plan* p) {
  int Q, RG;
  xpass_shape(p, &Q, &RG);
  return p->method != FD3_METHOD_EWALD && p->has_fft2 && p->precision == FD3_PREC_MIXED && p->mg.fft_x == 2 &&
         xpass_applies(p->mg, Q, RG);
}
// fused (y, z) transforms in effect: float mesh on a 2D-transform path, ny = nz = 256, asked for
static bool fft_yz_on(const fd3_plan* p) {
  return p->precision == FD3_PREC_MIXED && p->method != FD3_METHOD_EWALD && p->mg.fft_yz != 0 &&
         yzfft_applies(p->mg);
}
// cluster shape of the fused (y, z) forward transform: the knob, or pairs by default
static int yz_variant(const fd3_plan* p) { return p->mg.fft_yz > 0 ? p->mg.fft_yz : 1; }
static bool old_xpass_on(const fd3_plan* p) {
  return p->method != FD3_METHOD_EWALD && p->has_fft2 && p->mg.fft_x == 1 &&
         xfilter_pencil(p->mg, p->precision == FD3_PREC_FP64 ? 1 : 0) > 0;
}

extern "C" int fd3_plan_set_tuning(fd3_plan* p, int32_t knob, int32_t value) {
  if (!p) return FD3_EINVAL;
  if (knob == FD3_TUNE_FILTER_KT) {
    if (p->method == FD3_METHOD_EWALD) return FD3_OK;   // no mesh filter
    const size_t ts = p->precision == FD3_PREC_FP64 ? 8 : 4;
    if (value != -1 && !filter_kt_valid(value, p->S, p->R, ts)) {
      set_error("fd3_plan_set_tuning", "filter k-tile must be -1, 0 (<= 8 species) or 1/2/4/8/16 within shared memory");
      return FD3_EINVAL;
    }
    p->mg.filter_kt = value;
    return FD3_OK;
  }
  if (knob == FD3_TUNE_SPREAD_ZC) {
    if (value < -1 || value > 64) {
      set_error("fd3_plan_set_tuning", "spread z-chunk must be -1 (default), 0 (per-tile kernel) or 1..64");
      return FD3_EINVAL;
    }
    p->mg.spread_zc = value;
    return FD3_OK;
  }
  if (knob == FD3_TUNE_FFT_X) {
    if (value < -1 || value > 2) {
      set_error("fd3_plan_set_tuning", "fused x-pass must be -1 (default), 0 (3D FFT + filter), 1 or 2 (TMA)");
      return FD3_EINVAL;
    }
    p->mg.fft_x = value;
    return FD3_OK;
  }
  if (knob == FD3_TUNE_XQ) {
    if (value != -1 && value != 4 && value != 8 && value != 16 && value != 32) {
      set_error("fd3_plan_set_tuning", "TMA x-pass q values per unit must be -1 (default), 4, 8, 16 or 32");
      return FD3_EINVAL;
    }
    p->mg.xq = value;
    return FD3_OK;
  }
  if (knob == FD3_TUNE_XRANKS) {
    if (value != -1 && value != 1 && value != 2 && value != 4) {
      set_error("fd3_plan_set_tuning", "TMA x-pass ranks per unit must be -1 (default), 1, 2 or 4");
      return FD3_EINVAL;
    }
    p->mg.xranks = value;
    return FD3_OK;
  }
  if (knob == FD3_TUNE_FILTER_MMA) {
    if (value < -1 || value > 1) {
      set_error("fd3_plan_set_tuning", "tensor-core filter must be -1 (default), 0 (CUDA cores) or 1");
      return FD3_EINVAL;
    }
    p->mg.filter_mma = value;
    return FD3_OK;
  }
  if (knob == FD3_TUNE_XPENCIL) {
    if (value != -1 && value != 1 && value != 2 && value != 4) {
      set_error("fd3_plan_set_tuning", "fused x-pass pencil must be -1 (default), 1, 2 or 4 kz values");
      return FD3_EINVAL;
    }
    p->mg.xpencil = value;
    return FD3_OK;
  }
  if (knob == FD3_TUNE_FFT_YZ) {
    if (value < -1 || value > 2) {
      set_error("fd3_plan_set_tuning", "fused (y, z) transforms must be -1 (default), 0 (cuFFT), 1 or 2");
      return FD3_EINVAL;
    }
    p->mg.fft_yz = value;
    return FD3_OK;
  }
  if (knob == FD3_TUNE_GATHER_TILE) {
    if (value < -1 || value > 1) {
      set_error("fd3_plan_set_tuning", "tile-staged gather must be -1 (default), 0 (per-atom gather) or 1");
      return FD3_EINVAL;
    }
    p->mg.gather_tile = value;
    return FD3_OK;
  }
  if (knob == FD3_TUNE_SPREAD_CAP) {
    if (value != 0 && value < 256) {
      set_error("fd3_plan_set_tuning", "spread staging cap must be 0 (shared-memory bound) or >= 256");
      return FD3_EINVAL;
    }
    p->mg.spread_cap = value;
    return FD3_OK;
  }
  set_error("fd3_plan_set_tuning", "unknown knob");
  return FD3_EINVAL;
}

extern "C" int fd3_plan_get_tuning(const fd3_plan* p, int32_t knob, int32_t* value) {
  if (!p || !value) return FD3_EINVAL;
  if (knob == FD3_TUNE_FILTER_KT) {
    const size_t ts = p->precision == FD3_PREC_FP64 ? 8 : 4;
    *value = p->method == FD3_METHOD_EWALD ? -1
             : p->mg.filter_kt >= 0        ? p->mg.filter_kt
                                           : filter_default_kt(p->S, p->R, ts);
    return FD3_OK;
  }
  if (knob == FD3_TUNE_SPREAD_ZC) {
    *value = p->method == FD3_METHOD_EWALD ? -1
                                           : spread_chunk_in_effect(p->mg, p->precision == FD3_PREC_FP64 ? 8 : 4);
    return FD3_OK;
  }
  if (knob == FD3_TUNE_SPREAD_CAP) {
    *value = p->mg.spread_cap;
    return FD3_OK;
  }
  if (knob == FD3_TUNE_FFT_X) {
    *value = xpass_on(p) ? 2 : old_xpass_on(p) ? 1 : 0;
    return FD3_OK;
  }
  if (knob == FD3_TUNE_XQ || knob == FD3_TUNE_XRANKS) {
    int Q = 0, RG = 0;
    xpass_shape(p, &Q, &RG);
    const bool ok = p->has_fft2 && p->precision == FD3_PREC_MIXED && xpass_applies(p->mg, Q, RG);
    *value = ok ? (knob == FD3_TUNE_XQ ? Q : RG) : 0;
    return FD3_OK;
  }
  if (knob == FD3_TUNE_FILTER_MMA) {
    *value = p->method != FD3_METHOD_EWALD && p->precision == FD3_PREC_MIXED && !xpass_on(p) && !old_xpass_on(p) &&
                     filter_mma_on(p->mg)
                 ? 1
                 : 0;
    return FD3_OK;
  }
  if (knob == FD3_TUNE_XPENCIL) {
    *value = p->has_fft2 ? xfilter_pencil(p->mg, p->precision == FD3_PREC_FP64 ? 1 : 0) : 0;
    return FD3_OK;
  }
  if (knob == FD3_TUNE_FFT_YZ) {
    *value = (xpass_on(p) || old_xpass_on(p)) && fft_yz_on(p) ? yz_variant(p) : 0;
    return FD3_OK;
  }
  if (knob == FD3_TUNE_GATHER_TILE) {
    *value = p->method != FD3_METHOD_EWALD && p->mg.gather_tile == 1 &&
                     gather_tile_applies(p->mg, p->precision == FD3_PREC_FP64 ? 8 : 4)
                 ? 1
                 : 0;
    return FD3_OK;
  }
  set_error("fd3_plan_get_tuning", "unknown knob");
  return FD3_EINVAL;
}

extern "C" int fd3_plan_set_edge_cutoff(fd3_plan* p, int32_t on) {
  if (!p || (on != 0 && on != 1)) return FD3_EINVAL;
  p->edge_cutoff = on;
  return FD3_OK;
}

extern "C" int fd3_plan_destroy(fd3_plan* p) {
  if (!p) return FD3_OK;
  for (int k = 0; k < fd3_plan::kMaxMarks; ++k)
    if (p->ev[k]) cudaEventDestroy(p->ev[k]);
  if (p->fwd) cufftDestroy(p->fwd);
  if (p->inv) cufftDestroy(p->inv);
  if (p->fwd2) cufftDestroy(p->fwd2);
  if (p->fwd_cn) cufftDestroy(p->fwd_cn);
  if (p->inv_cn) cufftDestroy(p->inv_cn);
  cudaFree(p->d_cnpair);
  cudaFree(p->d_cnself);
  if (p->inv2) cufftDestroy(p->inv2);
  if (p->ev_fork) cudaEventDestroy(p->ev_fork);
  if (p->ev_join) cudaEventDestroy(p->ev_join);
  if (p->side) cudaStreamDestroy(p->side);
  cudaFree(p->d_tab);
  cudaFree(p->d_eigvecs);
  cudaFree(p->d_green);
  cudaFree(p->d_green_f);
  cudaFree(p->d_deconv);
  cudaFree(p->d_win_axes);
  delete p;
  return FD3_OK;
}

// ------------------------------------------------------------------ workspace layout
namespace {
struct Carver {
  size_t off = 0;
  char* base = nullptr;
  template <typename T>
  T* take(size_t count) {
    off = (off + 255) & ~(size_t)255;
    T* r = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += sizeof(T) * (count ? count : 1);
    return r;
  }
};

struct Work {
  CellInfo* ci;
  double *cn, *c6, *dc6, *gcn;
  double *self_part, *kspc_part, *cnv_part, *mcell_part;
  int *mkeys, *mcount, *mstart, *morder;
  MeshRecords rec;
  CellList cl;
  HitStore hits;
  EwaldWork ew;
  EdgeIndex ei;
  void *cn4_rho, *cn4_phi, *cn4_rhat, *cn4_spec;
  double *cn4_vals, *cn4_part;
  void *rho, *spec, *fftw;
  void* gtab;   // mixed-form Green table
};

// K = number of cell-list bins of the fused path, 0 for the edge-list path (no cell list);
// E = edges of the edge-list path.
void carve(const fd3_plan* p, int64_t N, int64_t K_in, Carver& c, Work& w, int64_t E = 0) {
  const bool fused = K_in > 0;
  const int64_t K = fused ? K_in : 1;
  const size_t es = p->precision == FD3_PREC_FP64 ? sizeof(double) : sizeof(float);
  const int R = p->R;
  // per-block partials: per-atom kernels use ceil(N/8) blocks, the bin kernels one per bin
  const int64_t nblk = (2 * ((N + 7) / 8) > K ? 2 * ((N + 7) / 8) : K) + 1;
  w.ci = c.take<CellInfo>(1);
  w.cn = c.take<double>(N);
  w.c6 = c.take<double>(N * R);
  w.dc6 = c.take<double>(N * R);
  w.gcn = c.take<double>(N);
  w.self_part = c.take<double>(nblk);
  w.cnv_part = c.take<double>(9 * nblk);
  // mesh-cell partials: one per gather CTA (atom warps or (tile, species) CTAs)
  int64_t ngt = 1;
  if (p->method != FD3_METHOD_EWALD) ngt = (int64_t)p->mg.nt[0] * p->mg.nt[1] * p->mg.nt[2] * p->S;
  // (+ the D4 CN gradient gather's blocks, appended after the dispersion gather's)
  const int64_t ncn4 = p->cnfunc == FD3_CN_D4 ? cn4_gather_blocks((int)N) : 0;
  w.mcell_part = c.take<double>(9 * ((nblk > ngt ? nblk : ngt) + ncn4 + 1));
  const bool mesh = p->method != FD3_METHOD_EWALD;
  size_t Mh = 0, M = 0;
  int64_t Kmesh = 1;
  if (mesh) {
    Mh = (size_t)p->mg.n[0] * p->mg.n[1] * p->mg.nzh;
    M = (size_t)p->mg.n[0] * p->mg.n[1] * p->mg.n[2];
    Kmesh = (int64_t)p->mg.nt[0] * p->mg.nt[1] * p->mg.nt[2] * p->S;
  }
  w.kspc_part = c.take<double>(7 * (filter_max_blocks() + 1));
  w.mkeys = c.take<int>(N);
  const size_t P3 = mesh ? (size_t)3 * p->P : 1;
  w.rec.b = c.take<int4>(N);
  w.rec.w = c.take<char>(N * P3 * es);
  w.rec.dw = c.take<char>(N * P3 * es);
  w.rec.c = c.take<char>(N * p->R * es);
  w.mcount = c.take<int>(Kmesh);
  w.mstart = c.take<int>(Kmesh + 1);
  w.morder = c.take<int>(N);
  w.cl.bin_of = c.take<int>(N);
  w.cl.bin_count = c.take<int>(K);
  w.cl.bin_start = c.take<int>(K + 1);
  w.cl.order = c.take<int>(N);
  w.cl.xs = c.take<double4>(N);
  w.cl.meta = c.take<int4>(N);
  w.cl.off = c.take<int4>(N);
  // CN pair records of the fused path
  const int64_t hn = fused ? N : 0;
  w.hits.cap = kHitCap;
  w.hits.is_double = p->precision == FD3_PREC_FP64;
  w.hits.j = c.take<int>(hn * kHitCap);
  w.hits.ad = c.take<char>(hn * kHitCap * 4 * es);
  w.hits.n = c.take<int>(N);
  w.hits.ovf = c.take<int>(1);
  const size_t C = (size_t)p->S * p->R;
  w.rho = c.take<char>(mesh ? C * M * es : 1);
  // the mixed form's spectrum may carry one pad slot per ky row (16-byte rows for the fused
  // (y, z) transforms under the TMA x-pass)
  const size_t Mh_spec = p->precision == FD3_PREC_MIXED ? Mh + (size_t)p->mg.n[0] * p->mg.n[1] : Mh;
  w.spec = c.take<char>(mesh ? C * Mh_spec * 2 * es : 1);
  w.fftw = c.take<char>(p->fft_ws);
  w.gtab = c.take<char>(mesh && p->precision == FD3_PREC_MIXED ? green_table_bytes(p->S) : 1);
  // D4 k-space CN: density / sigma / psi, phi, the density spectrum (kept for the adjoint), the
  // working spectrum, per-atom spread values and the strain partials
  const bool d4 = mesh && p->cnfunc == FD3_CN_D4;
  const size_t S_ = (size_t)p->S;
  w.cn4_rho = c.take<char>(d4 ? S_ * M * es : 1);
  w.cn4_phi = c.take<char>(d4 ? S_ * M * es : 1);
  w.cn4_rhat = c.take<char>(d4 ? S_ * Mh * 2 * es : 1);
  w.cn4_spec = c.take<char>(d4 ? S_ * Mh * 2 * es : 1);
  w.cn4_vals = c.take<double>(d4 ? N : 1);
  w.cn4_part = c.take<double>(d4 ? 9 * ((size_t)cn4_gather_blocks((int)N) + filter_max_blocks() + 2) : 1);
  // edge-list path: edges sorted by source and by destination
  w.ei.ks = c.take<int>(E);
  w.ei.kd = c.take<int>(E);
  w.ei.ord_s = c.take<int>(E);
  w.ei.ord_d = c.take<int>(E);
  w.ei.cnt = c.take<int>(N);
  w.ei.st_s = c.take<int>(N + 1);
  w.ei.st_d = c.take<int>(N + 1);
  w.ei.bad = c.take<int>(1);
  // direct Ewald sum
  if (!mesh) {
    const int64_t nk = (int64_t)p->ens[0] * p->ens[1] * p->ens[2];
    const int64_t nchunk = ewald_chunks((int)nk);
    w.ew.keys = c.take<int>(N);
    w.ew.counts = c.take<int>(p->S);
    w.ew.sp_start = c.take<int>(p->S + 1);
    w.ew.order = c.take<int>(N);
    w.ew.sp_of = c.take<int4>(N);
    w.ew.frac = c.take<double>(3 * N);
    w.ew.spec = c.take<char>((size_t)C * nk * 2 * es);
    w.ew.hspec = c.take<char>((size_t)C * nk * 2 * es);
    w.ew.kpart = w.kspc_part;
    w.ew.gpart = c.take<double>((size_t)N * nchunk * (p->R + 3));
  }
}
}  // namespace

extern "C" int fd3_workspace_size(const fd3_plan* p, int64_t n_atoms, int64_t n_bins, size_t* bytes) {
  if (!p || !bytes || n_atoms < 0) return FD3_EINVAL;
  Carver c;
  Work w;
  carve(p, n_atoms, n_bins > 0 ? n_bins : 0, c, w);
  *bytes = c.off + 256;
  return FD3_OK;
}

extern "C" int fd3_cell_grid(const double* h_cell, double r_cut, int32_t* nb3, int32_t* reach3) {
  CellGrid g;
  int rc = make_cell_grid(h_cell, r_cut, &g);
  if (rc) return rc;
  for (int a = 0; a < 3; ++a) {
    if (nb3) nb3[a] = g.nb[a];
    if (reach3) reach3[a] = g.reach[a];
  }
  return FD3_OK;
}

extern "C" int fd3_edge_workspace_size(const fd3_plan* p, int64_t n_atoms, int64_t n_edges, size_t* bytes) {
  if (!p || !bytes || n_atoms < 0 || n_edges < 0 || n_edges > INT32_MAX) return FD3_EINVAL;
  Carver c;
  Work w;
  carve(p, n_atoms, 0, c, w, n_edges);
  *bytes = c.off + 256;
  return FD3_OK;
}

static int check_work(const fd3_plan* p, int64_t N, int64_t K, void* work, size_t bytes, Work& w, int64_t E = 0) {
  Carver c;
  carve(p, N, K, c, w, E);
  if (!work || bytes < c.off + 256) {
    set_error("workspace", E > 0 ? "smaller than fd3_edge_workspace_size" : "smaller than fd3_workspace_size");
    return FD3_ENOMEM;
  }
  Carver c2;
  c2.base = reinterpret_cast<char*>(((uintptr_t)work + 255) & ~(uintptr_t)255);
  carve(p, N, K, c2, w, E);
  return FD3_OK;
}

// ------------------------------------------------------------------ shared mesh pipeline
// spread -> forward FFT -> filter (energy, virial, H = G S) -> [inverse FFT -> gather]
// atoms counting-sorted by (mesh tile, species): needs only the positions and the cell info
static int mesh_sort(fd3_plan* p, int N, const double* pos, double ps, const int32_t* species, Work& w,
                     cudaStream_t s) {
  const MeshGeom& mg = p->mg;
  const int Kmesh = mg.nt[0] * mg.nt[1] * mg.nt[2] * p->S;
  FD3_TRY(launch_mesh_keys(mg, N, pos, ps, species, w.ci, w.mkeys, s));
  return counting_sort(w.mkeys, N, Kmesh, w.mcount, w.mstart, w.morder, s);
}

// The position-only preparation of the mesh stage that can run beside the cell list and the CN
// stage: the stencil records' nodes and weights, and the mixed form's Green table.
static int mesh_side_prep(fd3_plan* p, int N, const double* pos, double ps, const int32_t* species, Work& w,
                          cudaStream_t s) {
  const MeshGeom& mg = p->mg;
  if (p->precision == FD3_PREC_FP64)
    return launch_spread<double>(mg, N, pos, ps, species, nullptr, w.ci, w.mstart, w.morder, w.rec, (double*)w.rho,
                                 s, kSpreadRecordsOnly);
  FD3_TRY(launch_spread<float>(mg, N, pos, ps, species, nullptr, w.ci, w.mstart, w.morder, w.rec, (float*)w.rho, s,
                               kSpreadRecordsOnly));
  return launch_green_table(mg, w.ci, p->d_green, p->d_tab, w.gtab, s);
}

template <typename T>
static int mesh_pipeline(fd3_plan* p, int N, const double* pos, double ps, const int32_t* species, Work& w,
                         bool need_grad, double* gpos, double* mcell, int* n_kspc, int* n_mcell, bool presorted,
                         cudaStream_t s, bool side_prep = false) {
  const MeshGeom& mg = p->mg;
  if (!presorted) FD3_TRY(mesh_sort(p, N, pos, ps, species, w, s));
  prof_mark(p, s, "mesh_sort");
  FD3_TRY(launch_spread<T>(mg, N, pos, ps, species, w.c6, w.ci, w.mstart, w.morder, w.rec, (T*)w.rho, s,
                           side_prep ? 1 : 0));
  prof_mark(p, s, "spread");
  const bool tma_x = sizeof(T) == 4 && xpass_on(p);
  if (tma_x || old_xpass_on(p)) {
    // the TMA x-pass between the fused (y, z) transforms: ky rows of nzh + 1 values (a zero pad
    // slot), so that the inverse transform can fetch its columns by TMA
    MeshGeom mgq = mg;
    mgq.qpitch = tma_x && sizeof(T) == 4 && fft_yz_on(p) && mg.nzh == 129 ? mg.nzh + 1 : mg.nzh;
    // (y, z) transforms by the fused cluster kernels or cuFFT; x transform, filter and inverse x
    // transform in one kernel
    const bool yz = sizeof(T) == 4 && fft_yz_on(p);
    if (yz) {
      FD3_TRY(launch_yz_forward(mgq, p->S * p->R, yz_variant(p), (const float*)w.rho, w.spec, s));
    } else {
      FD3_CUFFT(cufftSetStream(p->fwd2, s));
      FD3_CUFFT(cufftSetWorkArea(p->fwd2, w.fftw));
      if (sizeof(T) == 8)
        FD3_CUFFT(cufftExecD2Z(p->fwd2, (cufftDoubleReal*)w.rho, (cufftDoubleComplex*)w.spec));
      else
        FD3_CUFFT(cufftExecR2C(p->fwd2, (cufftReal*)w.rho, (cufftComplex*)w.spec));
    }
    prof_mark(p, s, "fft_r2c");
    if (sizeof(T) == 4 && !side_prep) FD3_TRY(launch_green_table(mg, w.ci, p->d_green, p->d_tab, w.gtab, s));
    if (tma_x) {
      int Q, RG;
      xpass_shape(p, &Q, &RG);
      FD3_TRY(launch_xpass(mgq, Q, RG, w.ci, p->d_green_f, (const float4*)w.gtab, p->d_tab, p->d_deconv,
                           p->method == FD3_METHOD_SPME, w.spec, w.kspc_part, n_kspc, s));
    } else {
      FD3_TRY(launch_xfilter<T>(mg, w.ci, p->d_green, p->d_green_f, (const float4*)w.gtab, p->d_tab, p->d_deconv,
                                p->method == FD3_METHOD_SPME, w.spec, w.kspc_part, n_kspc, s));
    }
    prof_mark(p, s, "filter");
    *n_mcell = 0;
    if (!need_grad) return FD3_OK;
    if (yz) {
      FD3_TRY(launch_yz_inverse(mgq, p->S * p->R, yz_variant(p), w.spec, (float*)w.rho, s));
    } else {
      FD3_CUFFT(cufftSetStream(p->inv2, s));
      FD3_CUFFT(cufftSetWorkArea(p->inv2, w.fftw));
      if (sizeof(T) == 8)
        FD3_CUFFT(cufftExecZ2D(p->inv2, (cufftDoubleComplex*)w.spec, (cufftDoubleReal*)w.rho));
      else
        FD3_CUFFT(cufftExecC2R(p->inv2, (cufftComplex*)w.spec, (cufftReal*)w.rho));
    }
    prof_mark(p, s, "fft_c2r");
    FD3_TRY(launch_gather<T>(mg, N, pos, ps, species, w.c6, w.dc6, w.ci, p->d_tab, w.morder, w.mstart, w.rec,
                             (const T*)w.rho, w.gcn, gpos, mcell, n_mcell, s));
    prof_mark(p, s, "gather");
    return FD3_OK;
  }
  FD3_CUFFT(cufftSetStream(p->fwd, s));
  FD3_CUFFT(cufftSetWorkArea(p->fwd, w.fftw));
  if (sizeof(T) == 8)
    FD3_CUFFT(cufftExecD2Z(p->fwd, (cufftDoubleReal*)w.rho, (cufftDoubleComplex*)w.spec));
  else
    FD3_CUFFT(cufftExecR2C(p->fwd, (cufftReal*)w.rho, (cufftComplex*)w.spec));
  prof_mark(p, s, "fft_r2c");
  void* hspec = w.spec;   // the filter overwrites the spectrum with H in place
  if (sizeof(T) == 4 && !side_prep) FD3_TRY(launch_green_table(mg, w.ci, p->d_green, p->d_tab, w.gtab, s));
  FD3_TRY(launch_filter<T>(mg, w.ci, p->d_green, p->d_green_f, (const float4*)w.gtab, p->d_tab, p->d_deconv, p->method == FD3_METHOD_SPME, w.spec,
                           w.kspc_part, n_kspc, s));
  prof_mark(p, s, "filter");
  *n_mcell = 0;
  if (!need_grad) return FD3_OK;
  FD3_CUFFT(cufftSetStream(p->inv, s));
  FD3_CUFFT(cufftSetWorkArea(p->inv, w.fftw));
  if (sizeof(T) == 8)
    FD3_CUFFT(cufftExecZ2D(p->inv, (cufftDoubleComplex*)hspec, (cufftDoubleReal*)w.rho));
  else
    FD3_CUFFT(cufftExecC2R(p->inv, (cufftComplex*)hspec, (cufftReal*)w.rho));
  prof_mark(p, s, "fft_c2r");
  FD3_TRY(launch_gather<T>(mg, N, pos, ps, species, w.c6, w.dc6, w.ci, p->d_tab, w.morder, w.mstart, w.rec,
                           (const T*)w.rho, w.gcn, gpos, mcell, n_mcell, s));
  prof_mark(p, s, "gather");
  return FD3_OK;
}

static int run_mesh(fd3_plan* p, int N, const double* pos, double ps, const int32_t* species, Work& w,
                    bool need_grad, double* gpos, double* mcell, int* n_kspc, int* n_mcell, cudaStream_t s,
                    bool presorted = false, bool side_prep = false) {
  if (p->method == FD3_METHOD_EWALD) {
    EwaldGeom eg{{p->ens[0], p->ens[1], p->ens[2]}, p->S, p->R};
    int rc;
    if (p->precision == FD3_PREC_FP64)
      rc = launch_ewald<double>(eg, N, pos, ps, species, w.c6, w.dc6, w.ci, p->d_green, p->d_tab, w.ew, need_grad,
                                w.gcn, gpos, mcell, n_kspc, n_mcell, s);
    else
      rc = launch_ewald<float>(eg, N, pos, ps, species, w.c6, w.dc6, w.ci, p->d_green, p->d_tab, w.ew, need_grad,
                               w.gcn, gpos, mcell, n_kspc, n_mcell, s);
    prof_mark(p, s, "ewald");
    return rc;
  }
  if (p->precision == FD3_PREC_FP64)
    return mesh_pipeline<double>(p, N, pos, ps, species, w, need_grad, gpos, mcell, n_kspc, n_mcell, presorted, s,
                                 side_prep);
  return mesh_pipeline<float>(p, N, pos, ps, species, w, need_grad, gpos, mcell, n_kspc, n_mcell, presorted, s,
                              side_prep);
}

// ------------------------------------------------------------------ D4 k-space CN stages
// Forward: one-hot species density -> 3D R2C (spectrum kept for the adjoint) -> G^CN -> C2R ->
// CN values (w.cn). Needs the mesh sort of this call (w.mstart, w.morder).
template <typename T>
static int cn4_forward(fd3_plan* p, int N, const double* pos, double ps, const int32_t* species, Work& w,
                       cudaStream_t s) {
  MeshGeom m1 = p->mg;
  m1.R = 1;
  const int spme = p->method == FD3_METHOD_SPME;
  FD3_TRY(launch_cn4_values(N, 0, nullptr, w.ci, w.cn4_vals, s));
  FD3_TRY(launch_spread<T>(m1, N, pos, ps, species, w.cn4_vals, w.ci, w.mstart, w.morder, w.rec, (T*)w.cn4_rho, s));
  FD3_CUFFT(cufftSetStream(p->fwd_cn, s));
  FD3_CUFFT(cufftSetWorkArea(p->fwd_cn, w.fftw));
  if (sizeof(T) == 8)
    FD3_CUFFT(cufftExecD2Z(p->fwd_cn, (cufftDoubleReal*)w.cn4_rho, (cufftDoubleComplex*)w.cn4_rhat));
  else
    FD3_CUFFT(cufftExecR2C(p->fwd_cn, (cufftReal*)w.cn4_rho, (cufftComplex*)w.cn4_rhat));
  int nb = 0;
  FD3_TRY(launch_cn4_filter<T>(p->mg, 0, w.ci, p->d_cnpair, p->d_deconv, spme, w.cn4_rhat, w.cn4_spec, nullptr, &nb,
                               s));
  FD3_CUFFT(cufftSetStream(p->inv_cn, s));
  FD3_CUFFT(cufftSetWorkArea(p->inv_cn, w.fftw));
  if (sizeof(T) == 8)
    FD3_CUFFT(cufftExecZ2D(p->inv_cn, (cufftDoubleComplex*)w.cn4_spec, (cufftDoubleReal*)w.cn4_phi));
  else
    FD3_CUFFT(cufftExecC2R(p->inv_cn, (cufftComplex*)w.cn4_spec, (cufftReal*)w.cn4_phi));
  return launch_cn4_gather<T>(p->mg, N, 0, pos, ps, w.ci, w.morder, w.rec, w.cn4_phi, nullptr, p->d_cnself, nullptr,
                              w.cn, nullptr, 0.0, nullptr, nullptr, s);
}

// Adjoint (after the dispersion gather has written dE/dCN to w.gcn): sigma spread -> R2C -> k-space
// strain partials and G^CN sigma -> C2R -> gradient gather: gpos = out_scale (gpos + dE/dx_CN),
// strain partials in w.cn4_part (*n_cnv blocks), positions-fixed cell partials appended to mcell.
template <typename T>
static int cn4_adjoint(fd3_plan* p, int N, const double* pos, double ps, const int32_t* species, Work& w,
                       double* gpos, double out_scale, double* mcell, int* n_cnv, cudaStream_t s) {
  MeshGeom m1 = p->mg;
  m1.R = 1;
  const int spme = p->method == FD3_METHOD_SPME;
  FD3_TRY(launch_cn4_values(N, 1, w.gcn, w.ci, w.cn4_vals, s));
  FD3_TRY(launch_spread<T>(m1, N, pos, ps, species, w.cn4_vals, w.ci, w.mstart, w.morder, w.rec, (T*)w.cn4_rho, s));
  FD3_CUFFT(cufftSetStream(p->fwd_cn, s));
  FD3_CUFFT(cufftSetWorkArea(p->fwd_cn, w.fftw));
  if (sizeof(T) == 8)
    FD3_CUFFT(cufftExecD2Z(p->fwd_cn, (cufftDoubleReal*)w.cn4_rho, (cufftDoubleComplex*)w.cn4_spec));
  else
    FD3_CUFFT(cufftExecR2C(p->fwd_cn, (cufftReal*)w.cn4_rho, (cufftComplex*)w.cn4_spec));
  const int nbg = cn4_gather_blocks(N);
  int nbf = 0;
  FD3_TRY(launch_cn4_filter<T>(p->mg, 1, w.ci, p->d_cnpair, p->d_deconv, spme, w.cn4_rhat, w.cn4_spec,
                               w.cn4_part + 9 * (size_t)nbg, &nbf, s));
  FD3_CUFFT(cufftSetStream(p->inv_cn, s));
  FD3_CUFFT(cufftSetWorkArea(p->inv_cn, w.fftw));
  if (sizeof(T) == 8)
    FD3_CUFFT(cufftExecZ2D(p->inv_cn, (cufftDoubleComplex*)w.cn4_spec, (cufftDoubleReal*)w.cn4_rho));
  else
    FD3_CUFFT(cufftExecC2R(p->inv_cn, (cufftComplex*)w.cn4_spec, (cufftReal*)w.cn4_rho));
  FD3_TRY(launch_cn4_gather<T>(p->mg, N, 1, pos, ps, w.ci, w.morder, w.rec, w.cn4_phi, w.cn4_rho, p->d_cnself, w.gcn,
                               w.cn, gpos, out_scale, w.cn4_part, mcell, s));
  *n_cnv = nbg + nbf;
  return FD3_OK;
}

static int cn4_forward_any(fd3_plan* p, int N, const double* pos, double ps, const int32_t* species, Work& w,
                           cudaStream_t s) {
  return p->precision == FD3_PREC_FP64 ? cn4_forward<double>(p, N, pos, ps, species, w, s)
                                       : cn4_forward<float>(p, N, pos, ps, species, w, s);
}
static int cn4_adjoint_any(fd3_plan* p, int N, const double* pos, double ps, const int32_t* species, Work& w,
                           double* gpos, double out_scale, double* mcell, int* n_cnv, cudaStream_t s) {
  return p->precision == FD3_PREC_FP64
             ? cn4_adjoint<double>(p, N, pos, ps, species, w, gpos, out_scale, mcell, n_cnv, s)
             : cn4_adjoint<float>(p, N, pos, ps, species, w, gpos, out_scale, mcell, n_cnv, s);
}

// ------------------------------------------------------------------ edge-list entry
extern "C" int fd3_energy_edges(fd3_plan* p, int64_t n_atoms, const double* d_pos, const int32_t* d_species,
                                const double* d_cell, int64_t n_edges, const int64_t* d_src, const int64_t* d_dst,
                                const double* d_shift, int32_t need_grad, void* d_work, size_t work_bytes,
                                double* d_energy, double* d_gpos, double* d_gshift, double* d_gcell, void* stream) {
  if (!p || n_atoms < 1 || n_atoms > (int64_t)1 << 30 || !d_pos || !d_species || !d_cell || !d_energy)
    return FD3_EINVAL;
  if (n_edges < 0 || n_edges > INT32_MAX || (n_edges > 0 && (!d_src || !d_dst || !d_shift))) return FD3_EINVAL;
  if (need_grad && (!d_gpos || !d_gcell || (n_edges > 0 && !d_gshift))) return FD3_EINVAL;
  cudaStream_t s = (cudaStream_t)stream;
  const int N = (int)n_atoms;
  Work w;
  FD3_TRY(check_work(p, N, 0, d_work, work_bytes, w, n_edges));
  prof_begin(p, s);
  FD3_TRY(launch_cellinfo(d_cell, 1.0, w.ci, s));
  if (p->cnfunc == FD3_CN_D4) {
    // k-space D4 CN: no edges (the reference's forward ignores them, core.py:512-516)
    int n_self = 0, n_kspc = 0, n_mcell = 0, n_cnv = 0;
    FD3_TRY(mesh_sort(p, N, d_pos, 1.0, d_species, w, s));
    FD3_TRY(cn4_forward_any(p, N, d_pos, 1.0, d_species, w, s));
    FD3_TRY(launch_c6_atoms(N, d_species, p->d_tab, p->d_eigvecs, p->R, w.cn, w.c6, w.dc6, w.self_part, &n_self, s));
    prof_mark(p, s, "cn_c6");
    FD3_TRY(run_mesh(p, N, d_pos, 1.0, d_species, w, need_grad != 0, d_gpos, w.mcell_part, &n_kspc, &n_mcell, s,
                     true));
    if (need_grad) {
      FD3_TRY(cn4_adjoint_any(p, N, d_pos, 1.0, d_species, w, d_gpos, 1.0, w.mcell_part + 9 * (size_t)n_mcell,
                              &n_cnv, s));
      n_mcell += cn4_gather_blocks(N);
    }
    prof_mark(p, s, "cn_adjoint");
    Partials pa{w.self_part, n_self, w.kspc_part, n_kspc, w.cn4_part, n_cnv, w.mcell_part, n_mcell};
    FD3_TRY(launch_finalize(pa, w.ci, 0, 1.0, d_energy, need_grad ? d_gcell : nullptr, s));
    prof_mark(p, s, "finalize");
    return FD3_OK;
  }
  // edges sorted by source and destination; the CN is summed per atom in edge order
  const double mask_r2 = p->edge_cutoff ? p->h_tab.r_cut * p->h_tab.r_cut : INFINITY;
  FD3_TRY(launch_edge_index(n_edges, N, d_src, d_dst, w.ei, s));
  FD3_TRY(launch_cn_edges_seg(n_edges, N, d_pos, d_species, d_src, d_dst, d_shift, p->d_tab, mask_r2, w.ei, w.cn,
                              s));
  int n_self = 0, n_kspc = 0, n_mcell = 0;
  FD3_TRY(launch_c6_atoms(N, d_species, p->d_tab, p->d_eigvecs, p->R, w.cn, w.c6, w.dc6, w.self_part, &n_self, s));
  prof_mark(p, s, "cn_c6");
  FD3_TRY(run_mesh(p, N, d_pos, 1.0, d_species, w, need_grad != 0, d_gpos, w.mcell_part, &n_kspc, &n_mcell, s));
  if (need_grad)
    FD3_TRY(launch_cn_adjoint_edges_seg(n_edges, N, d_pos, d_species, d_src, d_dst, d_shift, p->d_tab, mask_r2,
                                        w.gcn, w.ei, d_gpos, d_gshift, s));
  prof_mark(p, s, "cn_adjoint");
  Partials pa{w.self_part, n_self, w.kspc_part, n_kspc, w.cnv_part, 0, w.mcell_part, n_mcell};
  FD3_TRY(launch_finalize(pa, w.ci, 0, 1.0, d_energy, need_grad ? d_gcell : nullptr, s));
  prof_mark(p, s, "finalize");
  return FD3_OK;
}

// ------------------------------------------------------------------ fused entry
extern "C" int fd3_energy_forces_stress(fd3_plan* p, int64_t n_atoms, const double* d_pos_ang,
                                        const int32_t* d_species, const double* h_cell_ang,
                                        const double* d_cell_ang, double r_cut_ang, void* d_work,
                                        size_t work_bytes, double* d_energy, double* d_forces, double* d_stress,
                                        void* stream) {
  if (!p || n_atoms < 1 || n_atoms > (int64_t)1 << 30 || !d_pos_ang || !d_species || !h_cell_ang || !d_cell_ang ||
      !d_energy || !d_forces || !d_stress)
    return FD3_EINVAL;
  cudaStream_t s = (cudaStream_t)stream;
  const int N = (int)n_atoms;
  CellGrid g;
  FD3_TRY(make_cell_grid(h_cell_ang, r_cut_ang, &g));
  const int64_t K = (int64_t)g.nb[0] * g.nb[1] * g.nb[2];
  Work w;
  FD3_TRY(check_work(p, N, K, d_work, work_bytes, w));
  prof_begin(p, s);
  // the cell list below is built from the host cell: a device cell that differs (a captured graph
  // replayed after a cell change) makes every output NaN instead of silently dropping pairs
  FD3_TRY(launch_cellinfo(d_cell_ang, kAngToBohr, w.ci, s, p->cnfunc == FD3_CN_D4 ? nullptr : h_cell_ang));
  if (p->cnfunc == FD3_CN_D4) {
    // k-space D4 CN: no neighbour search (calculator.py:171-173)
    int n_self = 0, n_kspc = 0, n_mcell = 0, n_cnv = 0;
    FD3_TRY(mesh_sort(p, N, d_pos_ang, kAngToBohr, d_species, w, s));
    FD3_TRY(cn4_forward_any(p, N, d_pos_ang, kAngToBohr, d_species, w, s));
    FD3_TRY(launch_c6_atoms(N, d_species, p->d_tab, p->d_eigvecs, p->R, w.cn, w.c6, w.dc6, w.self_part, &n_self, s));
    prof_mark(p, s, "cn_c6");
    FD3_TRY(run_mesh(p, N, d_pos_ang, kAngToBohr, d_species, w, true, d_forces, nullptr, &n_kspc, &n_mcell, s,
                     true));
    FD3_TRY(cn4_adjoint_any(p, N, d_pos_ang, kAngToBohr, d_species, w, d_forces, -kHartreeToEv * kAngToBohr,
                            nullptr, &n_cnv, s));
    prof_mark(p, s, "cn_adjoint");
    Partials pa{w.self_part, n_self, w.kspc_part, n_kspc, w.cn4_part, n_cnv, nullptr, 0};
    FD3_TRY(launch_finalize(pa, w.ci, 1, kHartreeToEv, d_energy, d_stress, s));
    prof_mark(p, s, "finalize");
    return FD3_OK;
  }
  const bool fork = p->side != nullptr && p->method != FD3_METHOD_EWALD;
  if (fork) {   // mesh sort, stencil records and Green table on the side stream, beside the cell list and CN
    FD3_CUDA(cudaEventRecord(p->ev_fork, s));
    FD3_CUDA(cudaStreamWaitEvent(p->side, p->ev_fork, 0));
    FD3_TRY(mesh_sort(p, N, d_pos_ang, kAngToBohr, d_species, w, p->side));
    FD3_TRY(mesh_side_prep(p, N, d_pos_ang, kAngToBohr, d_species, w, p->side));
    FD3_CUDA(cudaEventRecord(p->ev_join, p->side));
  }
  FD3_TRY(build_cell_list(g, N, d_pos_ang, d_species, w.cl, s));
  prof_mark(p, s, "cell_list");
  int n_self = 0, n_kspc = 0, n_mcell = 0, n_cnv = 0;
  FD3_TRY(launch_cn_c6_cells(g, N, w.cl, d_pos_ang, d_species, p->d_tab, p->d_eigvecs, p->R, w.cn, w.c6, w.dc6,
                             w.self_part, &n_self, w.hits, s));
  prof_mark(p, s, "cn_c6");
  if (fork) FD3_CUDA(cudaStreamWaitEvent(s, p->ev_join, 0));
  // the mesh gradient (Hartree/Bohr) is staged in d_forces, then finished by the CN adjoint
  FD3_TRY(run_mesh(p, N, d_pos_ang, kAngToBohr, d_species, w, true, d_forces, nullptr, &n_kspc, &n_mcell, s,
                   fork, fork));
  FD3_TRY(launch_cn_adjoint_cells(g, N, w.cl, d_pos_ang, d_species, p->d_tab, w.gcn, d_forces,
                                  -kHartreeToEv * kAngToBohr, w.cnv_part, &n_cnv, w.hits, s));
  prof_mark(p, s, "cn_adjoint");
  Partials pa{w.self_part, n_self, w.kspc_part, n_kspc, w.cnv_part, n_cnv, nullptr, 0};
  FD3_TRY(launch_finalize(pa, w.ci, 1, kHartreeToEv, d_energy, d_stress, s));
  FD3_TRY(launch_poison_if_stale(w.ci, N, d_energy, d_forces, d_stress, s));
  prof_mark(p, s, "finalize");
  return FD3_OK;
}

// ------------------------------------------------------------------ direct pair sum (accuracy oracle)
namespace {
struct DirectWork {
  CellList cl;        // the bin grid of the pair cutoff r_direct
  double* dEdc;       // [N R]
  double* pair_part;  // [blocks 7]
  double* sp_part;    // [kDirSpBlocks S R]
  double* A;          // [S R]
  double* tail;       // [2]
  double* scratch;    // [S R + 2 S^2]: T, I_XY, phi_XY(Rc)
};
constexpr int kDirSpBlocks = 148;
void carve_direct(const fd3_plan* p, int64_t N, int64_t K2, Carver& c, DirectWork& d) {
  d.cl.bin_of = c.take<int>(N);
  d.cl.bin_count = c.take<int>(K2);
  d.cl.bin_start = c.take<int>(K2 + 1);
  d.cl.order = c.take<int>(N);
  d.cl.xs = c.take<double4>(N);
  d.cl.meta = c.take<int4>(N);
  d.cl.off = c.take<int4>(N);
  d.dEdc = c.take<double>((size_t)N * p->R);
  d.pair_part = c.take<double>((size_t)7 * ((N + 7) / 8));
  d.sp_part = c.take<double>((size_t)kDirSpBlocks * p->S * p->R);
  d.A = c.take<double>((size_t)p->S * p->R);
  d.tail = c.take<double>(2);
  d.scratch = c.take<double>(direct_scratch_doubles(p->S, p->R));
}
int direct_grids(const fd3_plan* p, int64_t N, const double* h_cell, double r_cut, double r_direct, CellGrid& g,
                 CellGrid& g2, size_t* fused_bytes, size_t* total_bytes) {
  if (!p || N < 1 || N > (int64_t)1 << 30 || !h_cell || !(r_direct > 0)) return FD3_EINVAL;
  if (p->cnfunc == FD3_CN_D4) {
    set_error("fd3_direct_energy_forces_stress", "the direct pair sum takes the smooth-cutoff CN");
    return FD3_EINVAL;
  }
  FD3_TRY(make_cell_grid(h_cell, r_cut, &g));
  FD3_TRY(make_cell_grid(h_cell, r_direct, &g2));
  Carver c;
  Work w;
  carve(p, N, (int64_t)g.nb[0] * g.nb[1] * g.nb[2], c, w);
  *fused_bytes = c.off;
  DirectWork d;
  carve_direct(p, N, (int64_t)g2.nb[0] * g2.nb[1] * g2.nb[2], c, d);
  *total_bytes = c.off + 512;
  return FD3_OK;
}
}  // namespace

extern "C" int fd3_direct_workspace_size(const fd3_plan* p, int64_t n_atoms, const double* h_cell_ang,
                                         double r_cut_ang, double r_direct_ang, size_t* bytes) {
  if (!bytes) return FD3_EINVAL;
  CellGrid g, g2;
  size_t fused = 0;
  return direct_grids(p, n_atoms, h_cell_ang, r_cut_ang, r_direct_ang, g, g2, &fused, bytes);
}

extern "C" int fd3_direct_energy_forces_stress(fd3_plan* p, int64_t n_atoms, const double* d_pos_ang,
                                               const int32_t* d_species, const double* h_cell_ang,
                                               const double* d_cell_ang, double r_cut_ang, double r_direct_ang,
                                               void* d_work, size_t work_bytes, double* d_energy, double* d_forces,
                                               double* d_stress, void* stream) {
  if (!d_pos_ang || !d_species || !d_cell_ang || !d_energy || !d_forces || !d_stress) return FD3_EINVAL;
  CellGrid g, g2;
  size_t fused = 0, total = 0;
  FD3_TRY(direct_grids(p, n_atoms, h_cell_ang, r_cut_ang, r_direct_ang, g, g2, &fused, &total));
  if (!d_work || work_bytes < total) {
    set_error("workspace", "smaller than fd3_direct_workspace_size");
    return FD3_ENOMEM;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int N = (int)n_atoms;
  Work w;
  FD3_TRY(check_work(p, N, (int64_t)g.nb[0] * g.nb[1] * g.nb[2], d_work, work_bytes, w));
  Carver c;   // the direct sum's buffers follow the fused ones
  c.base = reinterpret_cast<char*>(((uintptr_t)d_work + 255) & ~(uintptr_t)255);
  {
    Work skip;
    carve(p, N, (int64_t)g.nb[0] * g.nb[1] * g.nb[2], c, skip);
  }
  DirectWork d;
  carve_direct(p, N, (int64_t)g2.nb[0] * g2.nb[1] * g2.nb[2], c, d);
  FD3_TRY(launch_cellinfo(d_cell_ang, kAngToBohr, w.ci, s, h_cell_ang));
  FD3_TRY(build_cell_list(g, N, d_pos_ang, d_species, w.cl, s));
  int n_self = 0, n_pair = 0, n_cnv = 0;
  FD3_TRY(launch_cn_c6_cells(g, N, w.cl, d_pos_ang, d_species, p->d_tab, p->d_eigvecs, p->R, w.cn, w.c6, w.dc6,
                             w.self_part, &n_self, w.hits, s));
  FD3_TRY(build_cell_list(g2, N, d_pos_ang, d_species, d.cl, s));
  // pair gradient (Hartree/Bohr) staged in d_forces, finished by the CN adjoint
  FD3_TRY(launch_direct_pairs(g2, N, d.cl, w.c6, p->d_tab, p->R, p->S, p->d_green, d.dEdc, d_forces, d.pair_part,
                              &n_pair, s));
  FD3_TRY(launch_direct_tail_gcn(N, d_species, w.c6, w.dc6, d.dEdc, p->d_tab, p->d_green, p->S, p->R,
                                 r_direct_ang * kAngToBohr, w.ci, d.sp_part, kDirSpBlocks, d.A, d.tail, d.scratch,
                                 w.gcn, s));
  FD3_TRY(launch_cn_adjoint_cells(g, N, w.cl, d_pos_ang, d_species, p->d_tab, w.gcn, d_forces,
                                  -kHartreeToEv * kAngToBohr, w.cnv_part, &n_cnv, w.hits, s));
  FD3_TRY(launch_direct_finalize(d.pair_part, n_pair, d.tail, w.cnv_part, n_cnv, w.ci, d_energy, d_stress, s));
  FD3_TRY(launch_poison_if_stale(w.ci, N, d_energy, d_forces, d_stress, s));
  return FD3_OK;
}

// ------------------------------------------------------------------ per-atom read-back
extern "C" int fd3_atom_terms(const fd3_plan* p, int64_t n_atoms, int64_t n_bins, const void* d_work,
                              size_t work_bytes, double* d_cn, double* d_c6, void* stream) {
  if (!p || n_atoms < 1 || n_atoms > (int64_t)1 << 30 || n_bins < 0 || (!d_cn && !d_c6)) return FD3_EINVAL;
  Work w;
  FD3_TRY(check_work(p, n_atoms, n_bins, const_cast<void*>(d_work), work_bytes, w));
  cudaStream_t s = (cudaStream_t)stream;
  if (d_cn) FD3_CUDA(cudaMemcpyAsync(d_cn, w.cn, sizeof(double) * n_atoms, cudaMemcpyDeviceToDevice, s));
  if (d_c6)
    FD3_CUDA(cudaMemcpyAsync(d_c6, w.c6, sizeof(double) * n_atoms * p->R, cudaMemcpyDeviceToDevice, s));
  return FD3_OK;
}

// ------------------------------------------------------------------ neighbour export
namespace {
struct NbrWork {
  CellList cl;
  int* counts;
  int* row_start;
};
void carve_nbr(int64_t N, int64_t K, Carver& c, NbrWork& w) {
  w.cl.bin_of = c.take<int>(N);
  w.cl.bin_count = c.take<int>(K);
  w.cl.bin_start = c.take<int>(K + 1);
  w.cl.order = c.take<int>(N);
  w.cl.xs = c.take<double4>(N);
  w.cl.meta = c.take<int4>(N);
  w.cl.off = c.take<int4>(N);
  w.counts = c.take<int>(N);
  w.row_start = c.take<int>(N + 1);
}
int nbr_prepare(int64_t n, const double* d_pos, const double* h_cell, double r_cut, void* d_work, size_t bytes,
                CellGrid& g, NbrWork& w, cudaStream_t s) {
  if (n < 1 || n > (int64_t)1 << 30 || !d_pos || !h_cell) return FD3_EINVAL;
  FD3_TRY(make_cell_grid(h_cell, r_cut, &g));
  const int64_t K = (int64_t)g.nb[0] * g.nb[1] * g.nb[2];
  Carver c;
  carve_nbr(n, K, c, w);
  if (!d_work || bytes < c.off + 256) return FD3_ENOMEM;
  Carver c2;
  c2.base = reinterpret_cast<char*>(((uintptr_t)d_work + 255) & ~(uintptr_t)255);
  carve_nbr(n, K, c2, w);
  FD3_TRY(build_cell_list(g, (int)n, d_pos, nullptr, w.cl, s));
  FD3_TRY(launch_nbr_count(g, (int)n, w.cl, d_pos, w.counts, s));
  FD3_TRY(scan_exclusive(w.counts, (int)n, w.row_start, s));
  return FD3_OK;
}
}  // namespace

extern "C" int fd3_neighbor_workspace_size(int64_t n, const double* h_cell, double r_cut, size_t* bytes) {
  CellGrid g;
  if (!bytes || !h_cell || n < 1 || n > (int64_t)1 << 30) {
    set_error("fd3_neighbor_workspace_size", "need a cell, an output pointer and 1 <= n_atoms <= 2^30");
    return FD3_EINVAL;
  }
  FD3_TRY(make_cell_grid(h_cell, r_cut, &g));
  Carver c;
  NbrWork w;
  carve_nbr(n, (int64_t)g.nb[0] * g.nb[1] * g.nb[2], c, w);
  *bytes = c.off + 256;
  return FD3_OK;
}

extern "C" int fd3_neighbor_count(int64_t n, const double* d_pos, const double* h_cell, double r_cut, void* d_work,
                                  size_t bytes, int64_t* h_count, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  CellGrid g;
  NbrWork w;
  if (!h_count) return FD3_EINVAL;
  FD3_TRY(nbr_prepare(n, d_pos, h_cell, r_cut, d_work, bytes, g, w, s));
  int total = 0;
  FD3_CUDA(cudaMemcpyAsync(&total, w.row_start + n, sizeof(int), cudaMemcpyDeviceToHost, s));
  FD3_CUDA(cudaStreamSynchronize(s));
  *h_count = total;
  return FD3_OK;
}

extern "C" int fd3_neighbor_fill(int64_t n, const double* d_pos, const double* h_cell, double r_cut, void* d_work,
                                 size_t bytes, int64_t capacity, int64_t* d_src, int64_t* d_dst, int32_t* d_shift,
                                 int64_t* h_count, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  CellGrid g;
  NbrWork w;
  if (!h_count || !d_src || !d_dst || !d_shift) return FD3_EINVAL;
  FD3_TRY(nbr_prepare(n, d_pos, h_cell, r_cut, d_work, bytes, g, w, s));
  int total = 0;
  FD3_CUDA(cudaMemcpyAsync(&total, w.row_start + n, sizeof(int), cudaMemcpyDeviceToHost, s));
  FD3_CUDA(cudaStreamSynchronize(s));
  *h_count = total;
  if (total > capacity) return FD3_ECAPACITY;
  FD3_TRY(launch_nbr_fill(g, (int)n, w.cl, d_pos, w.row_start, d_src, d_dst, d_shift, s));
  return FD3_OK;
}

// ------------------------------------------------------------------ profiling
extern "C" int fd3_profile_enable(fd3_plan* p, int32_t on) {
  if (!p) return FD3_EINVAL;
  if (on && !p->ev[0])
    for (int k = 0; k < fd3_plan::kMaxMarks; ++k) FD3_CUDA(cudaEventCreate(&p->ev[k]));
  p->prof = on != 0;
  return FD3_OK;
}

extern "C" int fd3_profile_read(fd3_plan* p, double* ms, int32_t max_stages, char* names, int32_t names_len,
                                int32_t* n_stages) {
  if (!p || !ms || !n_stages) return FD3_EINVAL;
  *n_stages = 0;
  if (!p->prof || p->n_marks < 2) return FD3_OK;
  FD3_CUDA(cudaEventSynchronize(p->ev[p->n_marks - 1]));
  int n = 0;
  size_t used = 0;
  if (names && names_len > 0) names[0] = 0;
  for (int k = 1; k < p->n_marks && n < max_stages; ++k, ++n) {
    float t = 0.f;
    FD3_CUDA(cudaEventElapsedTime(&t, p->ev[k - 1], p->ev[k]));
    ms[n] = t;
    if (names && names_len > 0) {
      const int w = snprintf(names + used, names_len - used, "%s%s", n ? "," : "", p->mark_name[k]);
      if (w > 0 && used + w < (size_t)names_len) used += w;
    }
  }
  *n_stages = n;
  return FD3_OK;
}
