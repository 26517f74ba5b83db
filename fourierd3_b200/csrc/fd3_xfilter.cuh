// Fused x-pass: forward FFT along x, the reciprocal-space filter, inverse FFT along x.
//
// With this path cuFFT transforms only the (y, z) planes (batched 2D R2C / C2R over the C
// channels and nx planes); one kernel takes a pencil of the half spectrum -- one y, KZ
// consecutive kz, every x, every channel -- into shared memory, transforms it along x,
// filters every k-point of the pencil (the same per-k-point code as k_filter), transforms it
// back and writes it in place. The spectrum crosses HBM once between the two 2D transforms
// instead of three times (x pass, filter, x pass) on the 3D-FFT path. (cuFFT's 2D transforms
// with x innermost in the spectrum -- which would make each pencil one contiguous block --
// measured 3x slower than with the natural layout, so the pencil reads KZ-value pieces of
// the spectrum rows.)
//
// The x transform of length NX = N1 * N2 (N1, N2 in {8, 16}) is done in two register passes:
//   X[k1 + N1 k2] = sum_n2 w_N2^(n2 k2) w_NX^(n2 k1) [ sum_n1 x[N2 n1 + n2] w_N1^(n1 k1) ],
// each thread holding one N1- or N2-point DFT in registers (radix-2, static indices); the
// forward result is left in the (k1, k2) order and the inverse undoes the two passes in
// reverse, so no reordering pass is needed. A column is stored as N1 rows of N2 + 1 values
// (the padding keeps the row-wise and column-wise passes free of bank conflicts).
// Unnormalised in both directions, like cuFFT.
#pragma once
#include "fd3_filter.cuh"

namespace fd3 {

template <int N>
__host__ __device__ constexpr int brev_n(int i) {
  int r = 0;
  for (int b = 1, j = N >> 1; j; b <<= 1, j >>= 1)
    if (i & b) r |= j;
  return r;
}

template <int N>
__host__ __device__ constexpr int log2_n() {
  int l = 0;
  while ((1 << l) < N) ++l;
  return l;
}

// cos and sin of 2 pi m / 16, m in [0, 8)
__host__ __device__ constexpr double cos16(int m) {
  return m == 0 ? 1.0 : m == 1 ? 0.92387953251128675613 : m == 2 ? 0.70710678118654752440
       : m == 3 ? 0.38268343236508977173 : m == 4 ? 0.0 : m == 5 ? -0.38268343236508977173
       : m == 6 ? -0.70710678118654752440 : -0.92387953251128675613;
}
__host__ __device__ constexpr double sin16(int m) {
  return m == 0 ? 0.0 : m == 1 ? 0.38268343236508977173 : m == 2 ? 0.70710678118654752440
       : m == 3 ? 0.92387953251128675613 : m == 4 ? 1.0 : m == 5 ? 0.92387953251128675613
       : m == 6 ? 0.70710678118654752440 : 0.38268343236508977173;
}

// (br + i bi) * exp(SIGN 2 pi i m16 / 16), m16 a compile-time constant after unrolling
template <typename T, int SIGN>
__device__ __forceinline__ void cmul16(int m16, T br, T bi, T& tr, T& ti) {
  if (m16 == 0) {
    tr = br;
    ti = bi;
  } else if (m16 == 4) {   // SIGN i
    tr = -SIGN * bi;
    ti = SIGN * br;
  } else {
    const T c = (T)cos16(m16), sn = (T)(SIGN * sin16(m16));
    tr = br * c - bi * sn;
    ti = br * sn + bi * c;
  }
}

// In-register DFT of N <= 16 points, X[k] = sum_n x[n] exp(SIGN 2 pi i n k / N).
// Radix-2 decimation in time; every loop has a constant trip count, so after unrolling each
// index is a compile-time constant and the arrays stay in registers (a loop stepping by the
// stage length is not unrolled by nvcc and leaves the arrays in local memory).
template <typename T, int N, int SIGN>
__device__ __forceinline__ void dft_reg(T (&re)[N], T (&im)[N]) {
  T ar[N], ai[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    ar[brev_n<N>(i)] = re[i];
    ai[brev_n<N>(i)] = im[i];
  }
  constexpr int kLog = log2_n<N>();
#pragma unroll
  for (int st = 0; st < kLog; ++st) {   // butterflies of span 2^st, twiddle exp(SIGN 2 pi i j / 2^(st+1))
#pragma unroll
    for (int b = 0; b < N / 2; ++b) {
      const int j = b & ((1 << st) - 1);
      const int lo = ((b >> st) << (st + 1)) + j, hi = lo + (1 << st);
      T tr, ti;
      cmul16<T, SIGN>(j * (8 >> st), ar[hi], ai[hi], tr, ti);
      ar[hi] = ar[lo] - tr;
      ai[hi] = ai[lo] - ti;
      ar[lo] = ar[lo] + tr;
      ai[lo] = ai[lo] + ti;
    }
  }
#pragma unroll
  for (int i = 0; i < N; ++i) {
    re[i] = ar[i];
    im[i] = ai[i];
  }
}

// Asynchronous copies global -> shared; copy_async_wait_all waits for this thread's copies.
// One complex value (8 bytes through L1 for float, 16 bytes through L2 only for double):
template <typename C2>
__device__ __forceinline__ void copy_async(C2* dst, const C2* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(C2) == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
// 16 bytes (two float complex values), both addresses 16-byte aligned, through L2 only:
__device__ __forceinline__ void copy_async16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void copy_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_all;\n" ::: "memory");
}

template <int N1, int N2>
struct XLayout {
  static constexpr int NX = N1 * N2;
  static constexpr int ROW = N2 + 1;           // padded row (positions)
  static constexpr int PC = N1 * ROW;          // positions per column
  static constexpr int TW = N2 * (N1 + 1);     // twiddle table exp(-2 pi i n2 k1 / NX) at n2 (N1 + 1) + k1
  static constexpr int LN1 = log2_n<N1>(), LN2 = log2_n<N2>(), LNX = log2_n<NX>();
};

// Pencil layout in shared memory: for channel c, position p of the padded N1 x (N2 + 1) column
// and kz offset j, the value sits at c * (PC << LKZ) + (p << LKZ) + j -- the KZ values of one
// (c, x) are adjacent, as they are in the spectrum, so a pencil row moves in 16-byte copies.
template <typename T, int N1, int N2>
__host__ __device__ inline size_t xfilter_smem(int C, int KZ) {
  using L = XLayout<N1, N2>;
  return ((size_t)L::TW + (size_t)C * KZ * L::PC) * 2 * sizeof(T);
}

// Forward x transform of every column (c, j): natural order in, (k1, k2) order out.
template <typename T, int N1, int N2>
__device__ __forceinline__ void xfft_forward(typename Cplx<T>::type* buf, const typename Cplx<T>::type* tw, int C,
                                             int LKZ) {
  using C2 = typename Cplx<T>::type;
  using L = XLayout<N1, N2>;
  const int KZ = 1 << LKZ, CSC = L::PC << LKZ;
  // pass 1: lanes over (j, n2) -- a half-warp reads 16 adjacent values
  for (int it = threadIdx.x; it < (C * N2) << LKZ; it += blockDim.x) {
    const int j = it & (KZ - 1), n2 = (it >> LKZ) & (N2 - 1), c = it >> (LKZ + L::LN2);
    C2* b = buf + c * CSC + (n2 << LKZ) + j;
    T re[N1], im[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      const C2 v = b[(n1 * L::ROW) << LKZ];
      re[n1] = v.x;
      im[n1] = v.y;
    }
    dft_reg<T, N1, -1>(re, im);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
      const C2 w = tw[n2 * (N1 + 1) + k1];   // exp(-2 pi i n2 k1 / NX)
      b[(k1 * L::ROW) << LKZ] = C2{re[k1] * w.x - im[k1] * w.y, re[k1] * w.y + im[k1] * w.x};
    }
  }
  __syncthreads();
  // pass 2: lanes over (j, k1) -- rows (N2 + 1) << LKZ apart, free of bank conflicts
  for (int it = threadIdx.x; it < (C * N1) << LKZ; it += blockDim.x) {
    const int j = it & (KZ - 1), k1 = (it >> LKZ) & (N1 - 1), c = it >> (LKZ + L::LN1);
    C2* b = buf + c * CSC + ((k1 * L::ROW) << LKZ) + j;
    T re[N2], im[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) {
      const C2 v = b[n2 << LKZ];
      re[n2] = v.x;
      im[n2] = v.y;
    }
    dft_reg<T, N2, -1>(re, im);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) b[k2 << LKZ] = C2{re[k2], im[k2]};
  }
  __syncthreads();
}

// Inverse x transform: (k1, k2) order in, natural order out.
template <typename T, int N1, int N2>
__device__ __forceinline__ void xfft_inverse(typename Cplx<T>::type* buf, const typename Cplx<T>::type* tw, int C,
                                             int LKZ) {
  using C2 = typename Cplx<T>::type;
  using L = XLayout<N1, N2>;
  const int KZ = 1 << LKZ, CSC = L::PC << LKZ;
  for (int it = threadIdx.x; it < (C * N1) << LKZ; it += blockDim.x) {
    const int j = it & (KZ - 1), k1 = (it >> LKZ) & (N1 - 1), c = it >> (LKZ + L::LN1);
    C2* b = buf + c * CSC + ((k1 * L::ROW) << LKZ) + j;
    T re[N2], im[N2];
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) {
      const C2 v = b[k2 << LKZ];
      re[k2] = v.x;
      im[k2] = v.y;
    }
    dft_reg<T, N2, 1>(re, im);
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) b[n2 << LKZ] = C2{re[n2], im[n2]};
  }
  __syncthreads();
  for (int it = threadIdx.x; it < (C * N2) << LKZ; it += blockDim.x) {
    const int j = it & (KZ - 1), n2 = (it >> LKZ) & (N2 - 1), c = it >> (LKZ + L::LN2);
    C2* b = buf + c * CSC + (n2 << LKZ) + j;
    T re[N1], im[N1];
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
      const C2 v = b[(k1 * L::ROW) << LKZ];
      const C2 w = tw[n2 * (N1 + 1) + k1];   // conj: exp(+2 pi i n2 k1 / NX)
      re[k1] = v.x * w.x + v.y * w.y;
      im[k1] = v.y * w.x - v.x * w.y;
    }
    dft_reg<T, N1, 1>(re, im);
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) b[(n1 * L::ROW) << LKZ] = C2{re[n1], im[n1]};
  }
  __syncthreads();
}

// Pencil start along kz. With float values and an even number of values per spectrum x-row
// block (ny * (nz/2 + 1) even), every row of the pencil of one y starts at the same parity;
// shifting the pencil by that parity makes each pair of kz values one aligned 16-byte piece.
// Returns the first kz of pencil gz (-1 for the first pencil of a shifted y).
__device__ __forceinline__ int xpencil_start(int gz, int y, int nzh, int LKZ, bool pairs) {
  const int par = pairs ? ((y * nzh) & 1) : 0;
  return (gz << LKZ) - par;
}

// One CTA per pencil (y, kz0..kz0+KZ-1), KZ = 2^LKZ, at a time (grid-stride over pencils); the
// spectrum must hold the (y, z) 2D transforms of the C channels (layout (C, nx, ny, nz/2+1)).
// LKZ is a template parameter: constant shifts keep the float kernel within 80 registers.
template <typename T, int MAXS, int MAXR, int N1, int N2, int LKZ>
__global__ void __launch_bounds__(kFilterThreads, sizeof(T) == 4 && MAXS * MAXR <= 8 ? 3 : 1)
    k_xfilter(MeshDev g, int P, int spme, const CellInfo* __restrict__ ci,
              const typename GreenPairOf<T>::type* __restrict__ gp, const float4* __restrict__ gtab,
              const Tables* __restrict__ tab, const float* __restrict__ deconv,
              typename Cplx<T>::type* __restrict__ spec, double* __restrict__ part) {
  using C2 = typename Cplx<T>::type;
  using L = XLayout<N1, N2>;
  constexpr int NX = L::NX;
  extern __shared__ __align__(16) unsigned char xs_raw[];
  C2* tw = reinterpret_cast<C2*>(xs_raw);   // [n2][k1] exp(-2 pi i n2 k1 / NX), rows of N1 + 1
  C2* buf = tw + L::TW;                     // TW * sizeof(C2) is a multiple of 16 bytes
  const int KZ = 1 << LKZ;
  const int C = g.S * g.R;
  const int CSC = L::PC << LKZ;
  const int n1 = g.n[1], nzh = g.nzh;
  const size_t xrow = (size_t)n1 * nzh;   // values between consecutive x of one channel
  // float pencils of KZ >= 2 move as 16-byte pairs when every row of a pencil has one parity
  const bool pairs = sizeof(T) == 4 && LKZ >= 1 && (xrow & 1) == 0;
  for (int m = threadIdx.x; m < L::TW; m += blockDim.x) {
    const int a = m / (N1 + 1), b = m % (N1 + 1);
    double sn, cs;
    sincospi(-2.0 * ((a * b) % NX) / NX, &sn, &cs);
    tw[m] = C2{(T)cs, (T)sn};
  }
  const int ngz = (nzh + (pairs ? 1 : 0) + KZ - 1) >> LKZ;
  const int ngroups = n1 * ngz;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  const T s6 = (T)tab->s6, s8 = (T)tab->s8;
  T rc[9];
  load_recip<T>(ci, rc);
  float inv_h = 0.f;
  if constexpr (sizeof(T) == 4) inv_h = green_inv_h(g, ci);
  for (int grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    const int y = grp / ngz;
    const int kz0 = xpencil_start(grp - y * ngz, y, nzh, LKZ, pairs);
    const C2* src = spec + (size_t)y * nzh + kz0;   // + (c NX + x) xrow + j, valid for 0 <= kz0 + j < nzh
    __syncthreads();   // twiddles written; the previous pencil has been stored
    // every copy of the pencil is in flight at once (asynchronous global -> shared copies)
    if (pairs) {
      constexpr int LNV = LKZ >= 1 ? LKZ - 1 : 0;   // pairs per (c, x) = 2^LNV
      for (int i = threadIdx.x; i < (C * NX) << LNV; i += blockDim.x) {
        const int v = i & ((1 << LNV) - 1), cx = i >> LNV, c = cx >> L::LNX, x = cx & (NX - 1);
        const int kz = kz0 + 2 * v;
        C2* d = buf + c * CSC + (((x >> L::LN2) * L::ROW + (x & (N2 - 1))) << LKZ) + 2 * v;
        const C2* s = src + (size_t)cx * xrow + 2 * v;
        if (kz >= 0 && kz + 1 < nzh) {
          copy_async16(d, s);
        } else {   // ragged pencil ends
          d[0] = (kz >= 0 && kz < nzh) ? s[0] : C2{T(0), T(0)};
          d[1] = (kz + 1 < nzh) ? s[1] : C2{T(0), T(0)};
        }
      }
    } else {
      for (int i = threadIdx.x; i < (C * NX) << LKZ; i += blockDim.x) {
        const int j = i & (KZ - 1), cx = i >> LKZ, c = cx >> L::LNX, x = cx & (NX - 1);
        const int kz = kz0 + j;
        C2* d = buf + c * CSC + (((x >> L::LN2) * L::ROW + (x & (N2 - 1))) << LKZ) + j;
        if (kz < nzh)
          copy_async(d, src + (size_t)cx * xrow + j);
        else
          *d = C2{T(0), T(0)};
      }
    }
    copy_async_wait_all();
    __syncthreads();
    xfft_forward<T, N1, N2>(buf, tw, C, LKZ);
    for (int pt = threadIdx.x; pt < NX << LKZ; pt += blockDim.x) {
      const int j = pt & (KZ - 1), pos = pt >> LKZ;   // consecutive lanes: adjacent values
      const int iz = kz0 + j;
      if (iz < 0 || iz >= nzh) continue;
      const int k1 = pos >> L::LN2, k2 = pos & (N2 - 1);
      const int ix = k1 + N1 * k2;
      const size_t k = ((size_t)ix * n1 + y) * nzh + iz;
      const KPoint<T> q = kpoint_idx<T>(g, ix, y, iz, k, rc, deconv, spme, P);
      filter_point<T, MAXS, MAXR>(q, g.S, g.R, gp, gtab, inv_h, s6, s8, tab,
                                  buf + ((k1 * L::ROW + k2) << LKZ) + j, (size_t)CSC, acc);
    }
    __syncthreads();
    xfft_inverse<T, N1, N2>(buf, tw, C, LKZ);
    C2* dst = spec + (size_t)y * nzh + kz0;
    if (pairs) {
      constexpr int LNV = LKZ >= 1 ? LKZ - 1 : 0;
      for (int i = threadIdx.x; i < (C * NX) << LNV; i += blockDim.x) {
        const int v = i & ((1 << LNV) - 1), cx = i >> LNV, c = cx >> L::LNX, x = cx & (NX - 1);
        const int kz = kz0 + 2 * v;
        const C2* d = buf + c * CSC + (((x >> L::LN2) * L::ROW + (x & (N2 - 1))) << LKZ) + 2 * v;
        C2* s = dst + (size_t)cx * xrow + 2 * v;
        if (kz >= 0 && kz + 1 < nzh) {
          *reinterpret_cast<float4*>(s) = *reinterpret_cast<const float4*>(d);
        } else {
          if (kz >= 0 && kz < nzh) s[0] = d[0];
          if (kz + 1 < nzh) s[1] = d[1];
        }
      }
    } else {
      for (int i = threadIdx.x; i < (C * NX) << LKZ; i += blockDim.x) {
        const int j = i & (KZ - 1), cx = i >> LKZ, c = cx >> L::LNX, x = cx & (NX - 1);
        if (kz0 + j < nzh)
          dst[(size_t)cx * xrow + j] = buf[c * CSC + (((x >> L::LN2) * L::ROW + (x & (N2 - 1))) << LKZ) + j];
      }
    }
  }
  block_sum_store<7>(acc, part + 7 * blockIdx.x);
}

// kz values per pencil for this plan (0: the fused path does not apply). A requested width
// (mg.xpencil = 1, 2 or 4) is used when it fits in 200 KB of shared memory; otherwise, and by
// default, the widest pencil that leaves three CTAs per SM (float) or fits in 100 KB (double).
// Wider pencils move longer pieces of each spectrum row (measured on the 256^3 x 8-channel
// float mesh without the L2 prefetch hint: 1.28, 0.675 and 0.568 ms for 1, 2 and 4 kz values).
template <typename T>
inline int xfilter_kz(const MeshGeom& mg) {
  const int C = mg.S * mg.R;
  if (mg.S > 4 || mg.R > 8) return 0;
  int n1 = 0, n2 = 0;
  if (mg.n[0] == 64) n1 = 8, n2 = 8;
  else if (mg.n[0] == 128) n1 = 8, n2 = 16;
  else if (mg.n[0] == 256) n1 = 16, n2 = 16;
  else return 0;
  auto bytes = [&](int kz) { return (((size_t)n2 * (n1 + 1)) + (size_t)C * kz * n1 * (n2 + 1)) * 2 * sizeof(T); };
  if ((mg.xpencil == 1 || mg.xpencil == 2 || mg.xpencil == 4) && bytes(mg.xpencil) <= 200 * 1024) return mg.xpencil;
  const size_t cap = sizeof(T) == 4 ? 74 * 1024 : 100 * 1024;
  for (int kz = 4; kz >= 2; kz >>= 1)
    if (bytes(kz) <= cap) return kz;
  return bytes(1) <= 200 * 1024 ? 1 : 0;
}

}  // namespace fd3
