// Fused x-pass: forward FFT along x, the reciprocal-space filter, inverse FFT along x.
//
// With this path cuFFT transforms only the (y, z) planes (batched 2D R2C / C2R over the C
// channels and nx planes); one kernel takes a pencil of the half spectrum -- one y, KZ
// consecutive kz, every x, every channel -- into shared memory, transforms it along x,
// filters every k-point of the pencil (the same per-k-point code as k_filter), transforms it
// back and writes it in place. The spectrum crosses HBM once between the two 2D transforms
// instead of three times (x pass, filter, x pass) on the 3D-FFT path.
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
template <typename T, int N, int SIGN>
__device__ __forceinline__ void dft_reg(T (&re)[N], T (&im)[N]) {
  T ar[N], ai[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    ar[brev_n<N>(i)] = re[i];
    ai[brev_n<N>(i)] = im[i];
  }
#pragma unroll
  for (int st = 1; st <= log2_n<N>(); ++st) {
    const int len = 1 << st, half = len >> 1;
#pragma unroll
    for (int i = 0; i < N; i += len)
#pragma unroll
      for (int j = 0; j < half; ++j) {
        T tr, ti;
        cmul16<T, SIGN>(j * (16 / len), ar[i + j + half], ai[i + j + half], tr, ti);
        ar[i + j + half] = ar[i + j] - tr;
        ai[i + j + half] = ai[i + j] - ti;
        ar[i + j] = ar[i + j] + tr;
        ai[i + j] = ai[i + j] + ti;
      }
  }
#pragma unroll
  for (int i = 0; i < N; ++i) {
    re[i] = ar[i];
    im[i] = ai[i];
  }
}

template <int N1, int N2>
struct XLayout {
  static constexpr int NX = N1 * N2;
  static constexpr int ROW = N2 + 1;           // padded row
  static constexpr int CS = N1 * ROW + 1;      // column stride (complex values)
  static constexpr int TW = N2 * (N1 + 1);     // twiddle table exp(-2 pi i n2 k1 / NX) at n2 (N1 + 1) + k1
};

// shared memory: twiddle table + C * KZ columns
template <typename T, int N1, int N2>
__host__ __device__ inline size_t xfilter_smem(int C, int KZ) {
  using L = XLayout<N1, N2>;
  return ((size_t)L::TW + (size_t)C * KZ * L::CS) * 2 * sizeof(T);
}

// Forward x transform of the columns [0, ncol): natural order in, (k1, k2) order out.
template <typename T, int N1, int N2>
__device__ __forceinline__ void xfft_forward(typename Cplx<T>::type* buf, const typename Cplx<T>::type* tw, int ncol) {
  using C2 = typename Cplx<T>::type;
  using L = XLayout<N1, N2>;
  for (int it = threadIdx.x; it < ncol * N2; it += blockDim.x) {
    C2* b = buf + (size_t)(it / N2) * L::CS;
    const int n2 = it % N2;
    T re[N1], im[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      const C2 v = b[n1 * L::ROW + n2];
      re[n1] = v.x;
      im[n1] = v.y;
    }
    dft_reg<T, N1, -1>(re, im);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
      const C2 w = tw[n2 * (N1 + 1) + k1];   // exp(-2 pi i n2 k1 / NX)
      b[k1 * L::ROW + n2] = C2{re[k1] * w.x - im[k1] * w.y, re[k1] * w.y + im[k1] * w.x};
    }
  }
  __syncthreads();
  for (int it = threadIdx.x; it < ncol * N1; it += blockDim.x) {
    C2* b = buf + (size_t)(it / N1) * L::CS + (it % N1) * L::ROW;
    T re[N2], im[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) {
      const C2 v = b[n2];
      re[n2] = v.x;
      im[n2] = v.y;
    }
    dft_reg<T, N2, -1>(re, im);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) b[k2] = C2{re[k2], im[k2]};
  }
  __syncthreads();
}

// Inverse x transform: (k1, k2) order in, natural order out.
template <typename T, int N1, int N2>
__device__ __forceinline__ void xfft_inverse(typename Cplx<T>::type* buf, const typename Cplx<T>::type* tw, int ncol) {
  using C2 = typename Cplx<T>::type;
  using L = XLayout<N1, N2>;
  for (int it = threadIdx.x; it < ncol * N1; it += blockDim.x) {
    C2* b = buf + (size_t)(it / N1) * L::CS + (it % N1) * L::ROW;
    T re[N2], im[N2];
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) {
      const C2 v = b[k2];
      re[k2] = v.x;
      im[k2] = v.y;
    }
    dft_reg<T, N2, 1>(re, im);
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) b[n2] = C2{re[n2], im[n2]};
  }
  __syncthreads();
  for (int it = threadIdx.x; it < ncol * N2; it += blockDim.x) {
    C2* b = buf + (size_t)(it / N2) * L::CS;
    const int n2 = it % N2;
    T re[N1], im[N1];
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
      const C2 v = b[k1 * L::ROW + n2];
      const C2 w = tw[n2 * (N1 + 1) + k1];   // conj: exp(+2 pi i n2 k1 / NX)
      re[k1] = v.x * w.x + v.y * w.y;
      im[k1] = v.y * w.x - v.x * w.y;
    }
    dft_reg<T, N1, 1>(re, im);
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) b[n1 * L::ROW + n2] = C2{re[n1], im[n1]};
  }
  __syncthreads();
}

// One CTA per pencil (y, kz0..kz0+KZ-1) at a time (grid-stride over pencils); the spectrum
// must hold the (y, z) 2D transforms of the C channels (layout (C, nx, ny, nz/2+1)).
template <typename T, int MAXS, int MAXR, int N1, int N2>
__global__ void __launch_bounds__(kFilterThreads) k_xfilter(MeshDev g, int P, int spme, int LKZ,
                                                            const CellInfo* __restrict__ ci,
                                                            const typename GreenPairOf<T>::type* __restrict__ gp,
                                                            const float4* __restrict__ gtab,
                                                            const Tables* __restrict__ tab,
                                                            const float* __restrict__ deconv,
                                                            typename Cplx<T>::type* __restrict__ spec,
                                                            double* __restrict__ part) {
  using C2 = typename Cplx<T>::type;
  using L = XLayout<N1, N2>;
  constexpr int NX = L::NX;
  extern __shared__ __align__(16) unsigned char xs_raw[];
  C2* tw = reinterpret_cast<C2*>(xs_raw);   // [n2][k1] exp(-2 pi i n2 k1 / NX), rows of N1 + 1
  C2* buf = tw + L::TW;
  const int KZ = 1 << LKZ;
  const int C = g.S * g.R;
  const int ncol = C * KZ;
  const int n1 = g.n[1], nzh = g.nzh;
  for (int m = threadIdx.x; m < L::TW; m += blockDim.x) {
    const int a = m / (N1 + 1), b = m % (N1 + 1);
    double sn, cs;
    sincospi(-2.0 * ((a * b) % NX) / NX, &sn, &cs);
    tw[m] = C2{(T)cs, (T)sn};
  }
  const int ngz = (nzh + KZ - 1) / KZ;
  const int ngroups = n1 * ngz;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  const T s6 = (T)tab->s6, s8 = (T)tab->s8;
  T rc[9];
  load_recip<T>(ci, rc);
  float inv_h = 0.f;
  if constexpr (sizeof(T) == 4) inv_h = green_inv_h(g, ci);
  for (int grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    const int y = grp / ngz, kz0 = (grp % ngz) * KZ;
    __syncthreads();   // twiddles written; the previous pencil has been stored
    for (int e = threadIdx.x; e < (C * NX) << LKZ; e += blockDim.x) {
      const int j = e & (KZ - 1), cx = e >> LKZ, x = cx % NX, c = cx / NX;
      const int iz = kz0 + j;
      buf[(size_t)(c * KZ + j) * L::CS + (x / N2) * L::ROW + (x % N2)] =
          iz < nzh ? spec[((size_t)cx * n1 + y) * nzh + iz] : C2{T(0), T(0)};
    }
    __syncthreads();
    xfft_forward<T, N1, N2>(buf, tw, ncol);
    for (int pt = threadIdx.x; pt < NX << LKZ; pt += blockDim.x) {
      const int j = pt / NX, pos = pt % NX;   // consecutive lanes: consecutive positions of one column
      const int iz = kz0 + j;
      if (iz >= nzh) continue;
      const int k1 = pos / N2, k2 = pos % N2;
      const int ix = k1 + N1 * k2;
      const size_t k = ((size_t)ix * n1 + y) * nzh + iz;
      const KPoint<T> q = kpoint_idx<T>(g, ix, y, iz, k, rc, deconv, spme, P);
      filter_point<T, MAXS, MAXR>(q, g.S, g.R, gp, gtab, inv_h, s6, s8, tab,
                                  buf + (size_t)j * L::CS + k1 * L::ROW + k2, (size_t)KZ * L::CS, acc);
    }
    __syncthreads();
    xfft_inverse<T, N1, N2>(buf, tw, ncol);
    for (int e = threadIdx.x; e < (C * NX) << LKZ; e += blockDim.x) {
      const int j = e & (KZ - 1), cx = e >> LKZ, x = cx % NX, c = cx / NX;
      const int iz = kz0 + j;
      if (iz < nzh)
        spec[((size_t)cx * n1 + y) * nzh + iz] = buf[(size_t)(c * KZ + j) * L::CS + (x / N2) * L::ROW + (x % N2)];
    }
  }
  block_sum_store<7>(acc, part + 7 * blockIdx.x);
}

// pencil width along kz for this plan (0: the fused path does not apply)
template <typename T>
inline int xfilter_kz(const MeshGeom& mg) {
  const int C = mg.S * mg.R;
  if (mg.S > 4 || mg.R > 8) return 0;
  int n1 = 0, n2 = 0;
  if (mg.n[0] == 64) n1 = 8, n2 = 8;
  else if (mg.n[0] == 128) n1 = 8, n2 = 16;
  else if (mg.n[0] == 256) n1 = 16, n2 = 16;
  else return 0;
  for (int kz = 4; kz >= 1; kz >>= 1) {
    const size_t b = (((size_t)n2 * (n1 + 1)) + (size_t)C * kz * (n1 * (n2 + 1) + 1)) * 2 * sizeof(T);
    if (b <= 100 * 1024) return kz;
  }
  return 0;
}

}  // namespace fd3
