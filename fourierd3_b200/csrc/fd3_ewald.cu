// Direct Ewald k-sum (reference: src/fourierd3/core.py:225-242, 563-577).
//
// k-vectors: the full Miller box of torch-pme's generate_kvectors_for_ewald, m_a in fftfreq order
// on every axis (k = 0 included), k = m0 b0 + m1 b1 + m2 b2. The reference weights rank r by
// sqrt(|lambda_r|) on both structure factors, i.e. the k-space energy uses |lambda_r| (the self
// term keeps the signed lambda_r); this is reproduced as is.
//
//   sf     : one thread per k; atoms (species-sorted) staged in shared memory; S_X^r(k) =
//            sum_{i in X} c_ir exp(i k.x_i) with the phase evaluated in turns, k.x = 2 pi m.s
//            (s = fractional coordinate), so sincospi stays accurate for any |k.x|.
//   filter : one thread per k; G_XY(|k|), energy and virial (float64 accumulation), H = G S.
//   gather : one thread per (atom, chunk of k); partial sums reduced per atom in a fixed order.
#include <math.h>

#include "fd3_internal.h"

namespace fd3 {

struct EwaldDev {
  int ns[3];
  int nk;
  int S, R;
};

__device__ __forceinline__ int fftfreq_order(int i, int n) { return i <= (n - 1) / 2 ? i : i - n; }

__device__ __forceinline__ void ewald_miller(const EwaldDev& e, int k, int& m0, int& m1, int& m2) {
  const int i2 = k % e.ns[2];
  const int i1 = (k / e.ns[2]) % e.ns[1];
  const int i0 = k / (e.ns[2] * e.ns[1]);
  m0 = fftfreq_order(i0, e.ns[0]);
  m1 = fftfreq_order(i1, e.ns[1]);
  m2 = fftfreq_order(i2, e.ns[2]);
}

template <typename T> struct Cplx2;
template <> struct Cplx2<double> { using type = double2; };
template <> struct Cplx2<float> { using type = float2; };

// fractional coordinates s = x inv(cell) of every atom, in species-sorted order
__global__ void __launch_bounds__(256) k_ewald_prep(int n, const double* __restrict__ pos, double ps,
                                                   const CellInfo* __restrict__ ci, const int* __restrict__ order,
                                                   double* __restrict__ frac) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = order[t];
  const double x0 = pos[3 * i] * ps, x1 = pos[3 * i + 1] * ps, x2 = pos[3 * i + 2] * ps;
#pragma unroll
  for (int a = 0; a < 3; ++a) frac[3 * t + a] = x0 * ci->inv[a] + x1 * ci->inv[3 + a] + x2 * ci->inv[6 + a];
}

constexpr int kEwTile = 128;

template <typename T, int MAXR>
__global__ void __launch_bounds__(256) k_ewald_sf(EwaldDev e, const double* __restrict__ frac,
                                                 const int* __restrict__ order, const int* __restrict__ sp_start,
                                                 const double* __restrict__ c6,
                                                 typename Cplx2<T>::type* __restrict__ spec) {
  using C2 = typename Cplx2<T>::type;
  __shared__ double s_f[kEwTile][3];
  __shared__ T s_c[kEwTile][MAXR];
  const int R = e.R;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  int m0 = 0, m1 = 0, m2 = 0;
  if (k < e.nk) ewald_miller(e, k, m0, m1, m2);
  for (int X = 0; X < e.S; ++X) {
    double are[MAXR], aim[MAXR];   // per-atom terms in T, accumulated in float64
#pragma unroll
    for (int r = 0; r < MAXR; ++r) are[r] = aim[r] = 0.0;
    const int a0 = sp_start[X], a1 = sp_start[X + 1];
    for (int t0 = a0; t0 < a1; t0 += kEwTile) {
      const int cnt = min(kEwTile, a1 - t0);
      __syncthreads();
      for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
        const int t = t0 + q;
        s_f[q][0] = frac[3 * t];
        s_f[q][1] = frac[3 * t + 1];
        s_f[q][2] = frac[3 * t + 2];
        const int i = order[t];
#pragma unroll
        for (int r = 0; r < MAXR; ++r) s_c[q][r] = r < R ? (T)c6[(size_t)i * R + r] : T(0);
      }
      __syncthreads();
      if (k < e.nk) {
        for (int q = 0; q < cnt; ++q) {
          // k.x / (2 pi) = m . s ; keep only the fractional part, then sin/cos of 2 pi * frac
          const double turns = m0 * s_f[q][0] + m1 * s_f[q][1] + m2 * s_f[q][2];
          const T fr = (T)(turns - rint(turns));
          T sn, cs;
          sincospi_t(T(2) * fr, &sn, &cs);
#pragma unroll
          for (int r = 0; r < MAXR; ++r) {
            are[r] += (double)(s_c[q][r] * cs);
            aim[r] += (double)(s_c[q][r] * sn);
          }
        }
      }
    }
    if (k < e.nk) {
#pragma unroll
      for (int r = 0; r < MAXR; ++r)
        if (r < R) spec[((size_t)X * R + r) * e.nk + k] = C2{(T)are[r], (T)aim[r]};
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_ewald_filter(EwaldDev e, const CellInfo* __restrict__ ci,
                                                     const GreenPair* __restrict__ gp, const Tables* __restrict__ tab,
                                                     typename Cplx2<T>::type* __restrict__ spec,
                                                     typename Cplx2<T>::type* __restrict__ hout,
                                                     double* __restrict__ part) {
  using C2 = typename Cplx2<T>::type;
  const int S = e.S, R = e.R;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  const T s6 = (T)tab->s6, s8 = (T)tab->s8;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < e.nk; k += gridDim.x * blockDim.x) {
    int m0, m1, m2;
    ewald_miller(e, k, m0, m1, m2);
    double kv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) kv[c] = m0 * ci->recip[c] + m1 * ci->recip[3 + c] + m2 * ci->recip[6 + c];
    const double knorm = sqrt(kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2]);
    double qq = 0.0, dq = 0.0;
    for (int X = 0; X < S; ++X) {
      for (int r = 0; r < R; ++r) {
        const size_t ix = ((size_t)X * R + r) * e.nk + k;
        const C2 sx = spec[ix];
        T hre = T(0), him = T(0), dre = T(0), dim = T(0);
        for (int Y = 0; Y < S; ++Y) {
          T gv, dv;
          green_eval<T>(gp[X * S + Y], (T)knorm, s6, s8, gv, dv);
          const C2 sy = spec[((size_t)Y * R + r) * e.nk + k];
          hre += gv * sy.x;
          him += gv * sy.y;
          dre += dv * sy.x;
          dim += dv * sy.y;
        }
        const double lam = fabs(tab->eigs[r]);
        qq += lam * ((double)sx.x * hre + (double)sx.y * him);
        dq += lam * ((double)sx.x * dre + (double)sx.y * dim);
        hout[ix] = C2{hre, him};
      }
    }
    acc[0] += qq;
    if (knorm > 0.0) {
      const double f = dq / knorm;
      acc[1] += f * kv[0] * kv[0];
      acc[2] += f * kv[1] * kv[1];
      acc[3] += f * kv[2] * kv[2];
      acc[4] += f * kv[0] * kv[1];
      acc[5] += f * kv[0] * kv[2];
      acc[6] += f * kv[1] * kv[2];
    }
  }
  block_sum_store<7>(acc, part + 7 * blockIdx.x);
}

constexpr int kEwChunk = 2048;   // k-points per gather thread

// Partial sums of one atom over one chunk of k: P_r = sum_k Re(e^{i phi} conj H_r) and
// U = sum_k k sum_r |lambda_r| c_r (-sin phi H_r.re + cos phi H_r.im)  (phi = k.x).
template <typename T, int MAXR>
__global__ void __launch_bounds__(256) k_ewald_gather(EwaldDev e, int n, const double* __restrict__ frac,
                                                     const int* __restrict__ order, const int4* __restrict__ sp_of,
                                                     const double* __restrict__ c6, const CellInfo* __restrict__ ci,
                                                     const Tables* __restrict__ tab,
                                                     const typename Cplx2<T>::type* __restrict__ h,
                                                     double* __restrict__ gpart, int nchunk) {
  using C2 = typename Cplx2<T>::type;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;    // atom slot (species-sorted)
  const int chunk = blockIdx.y;
  const int R = e.R;
  if (t >= n) return;
  const int i = order[t];
  const int X = sp_of[t].x;
  const double s0 = frac[3 * t], s1 = frac[3 * t + 1], s2 = frac[3 * t + 2];
  T cl[MAXR];
#pragma unroll
  for (int r = 0; r < MAXR; ++r) cl[r] = r < R ? (T)(c6[(size_t)i * R + r] * fabs(tab->eigs[r])) : T(0);
  double pr[MAXR];
#pragma unroll
  for (int r = 0; r < MAXR; ++r) pr[r] = 0.0;
  double u0 = 0, u1 = 0, u2 = 0;
  const int k0 = chunk * kEwChunk, k1 = min(e.nk, k0 + kEwChunk);
  for (int k = k0; k < k1; ++k) {
    int m0, m1, m2;
    ewald_miller(e, k, m0, m1, m2);
    const double turns = m0 * s0 + m1 * s1 + m2 * s2;
    const T fr = (T)(turns - rint(turns));
    T sn, cs;
    sincospi_t(T(2) * fr, &sn, &cs);
    T u = T(0);
#pragma unroll
    for (int r = 0; r < MAXR; ++r) {
      if (r < R) {
        const C2 hv = h[((size_t)X * R + r) * e.nk + k];
        pr[r] += (double)(cs * hv.x + sn * hv.y);
        u += cl[r] * (-sn * hv.x + cs * hv.y);
      }
    }
    // u multiplies the Cartesian k = m0 b0 + m1 b1 + m2 b2; accumulate per Miller axis
    u0 += (double)u * m0;
    u1 += (double)u * m1;
    u2 += (double)u * m2;
  }
  double* out = gpart + ((size_t)t * nchunk + chunk) * (R + 3);
  for (int r = 0; r < R; ++r) out[r] = pr[r];
  out[R] = u0;
  out[R + 1] = u1;
  out[R + 2] = u2;
}

// Per atom: reduce the chunks in order, then dE/dc -> dE/dCN, the force and the cell term.
__global__ void __launch_bounds__(256) k_ewald_finish(EwaldDev e, int n, const double* __restrict__ frac,
                                                     const int* __restrict__ order, const int4* __restrict__ sp_of,
                                                     const double* __restrict__ c6, const double* __restrict__ dc6,
                                                     const CellInfo* __restrict__ ci, const Tables* __restrict__ tab,
                                                     const double* __restrict__ gpart, int nchunk,
                                                     double* __restrict__ gcn, double* __restrict__ gpos,
                                                     double* __restrict__ mcell_part) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int R = e.R;
  double mc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (t < n) {
    const int i = order[t];
    const int X = sp_of[t].x;
    double pr[FD3_MAX_RANK + 3];
    for (int q = 0; q < R + 3; ++q) pr[q] = 0.0;
    for (int c = 0; c < nchunk; ++c) {
      const double* src = gpart + ((size_t)t * nchunk + c) * (R + 3);
      for (int q = 0; q < R + 3; ++q) pr[q] += src[q];
    }
    const double inv_vol = 1.0 / ci->volume;
    double gsum = 0.0;
    for (int r = 0; r < R; ++r) {
      const double lam = tab->eigs[r];
      const double c = c6[(size_t)i * R + r];
      gsum += (-fabs(lam) * inv_vol * pr[r] + lam * c * tab->selfcont[X]) * dc6[(size_t)i * R + r];
    }
    // dE/dx = -(1/Omega) sum_k k (...) with k = sum_a m_a b_a  ->  -(1/Omega) sum_a U_a b_a
    double gx[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      gx[c] = -inv_vol * (pr[R] * ci->recip[c] + pr[R + 1] * ci->recip[3 + c] + pr[R + 2] * ci->recip[6 + c]);
    gcn[i] = gsum;
    gpos[3 * i] = gx[0];
    gpos[3 * i + 1] = gx[1];
    gpos[3 * i + 2] = gx[2];
    if (mcell_part) {
#pragma unroll
      for (int A = 0; A < 3; ++A)
#pragma unroll
        for (int a = 0; a < 3; ++a) mc[3 * A + a] = frac[3 * t + A] * gx[a];
    }
  }
  if (mcell_part) block_sum_store<9>(mc, mcell_part + 9 * blockIdx.x);
}

__global__ void __launch_bounds__(256) k_species_keys(int n, const int32_t* __restrict__ species,
                                                     int* __restrict__ keys) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) keys[i] = species[i];
}

__global__ void __launch_bounds__(256) k_species_of_slot(int n, const int* __restrict__ order,
                                                        const int32_t* __restrict__ species, int4* __restrict__ sp_of) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) sp_of[t] = make_int4(species[order[t]], 0, 0, 0);
}

int ewald_chunks(int nk) { return (nk + kEwChunk - 1) / kEwChunk; }

template <typename T>
int launch_ewald(const EwaldGeom& eg, int n, const double* pos, double ps, const int32_t* species,
                 const double* c6, const double* dc6, const CellInfo* ci, const GreenPair* gp, const Tables* tab,
                 const EwaldWork& w, bool need_grad, double* gcn, double* gpos, double* mcell_part, int* n_kspc,
                 int* n_mcell, cudaStream_t s) {
  using C2 = typename Cplx2<T>::type;
  EwaldDev e;
  for (int a = 0; a < 3; ++a) e.ns[a] = eg.ns[a];
  e.nk = eg.ns[0] * eg.ns[1] * eg.ns[2];
  e.S = eg.S;
  e.R = eg.R;
  if (e.R > FD3_MAX_RANK) return FD3_EINVAL;
  const int tb = 256;
  // species-sorted atom order
  k_species_keys<<<(n + tb - 1) / tb, tb, 0, s>>>(n, species, w.keys);
  FD3_LAUNCHED();
  int rc = counting_sort(w.keys, n, e.S, w.counts, w.sp_start, w.order, s);
  if (rc) return rc;
  k_species_of_slot<<<(n + tb - 1) / tb, tb, 0, s>>>(n, w.order, species, w.sp_of);
  FD3_LAUNCHED();
  k_ewald_prep<<<(n + tb - 1) / tb, tb, 0, s>>>(n, pos, ps, ci, w.order, w.frac);
  FD3_LAUNCHED();
  const int kb = (e.nk + tb - 1) / tb;
  C2* spec = reinterpret_cast<C2*>(w.spec);
  C2* hsp = reinterpret_cast<C2*>(w.hspec);
  if (e.R <= 4)
    k_ewald_sf<T, 4><<<kb, tb, 0, s>>>(e, w.frac, w.order, w.sp_start, c6, spec);
  else if (e.R <= 8)
    k_ewald_sf<T, 8><<<kb, tb, 0, s>>>(e, w.frac, w.order, w.sp_start, c6, spec);
  else if (e.R <= 16)
    k_ewald_sf<T, 16><<<kb, tb, 0, s>>>(e, w.frac, w.order, w.sp_start, c6, spec);
  else
    k_ewald_sf<T, 32><<<kb, tb, 0, s>>>(e, w.frac, w.order, w.sp_start, c6, spec);
  FD3_LAUNCHED();
  const int fb = kb < 148 * 8 ? kb : 148 * 8;
  k_ewald_filter<T><<<fb, tb, 0, s>>>(e, ci, gp, tab, spec, hsp, w.kpart);
  FD3_LAUNCHED();
  *n_kspc = fb;
  *n_mcell = 0;
  if (!need_grad) return FD3_OK;
  const int nchunk = ewald_chunks(e.nk);
  const dim3 gg((n + tb - 1) / tb, nchunk);
  if (e.R <= 4)
    k_ewald_gather<T, 4><<<gg, tb, 0, s>>>(e, n, w.frac, w.order, w.sp_of, c6, ci, tab, hsp, w.gpart, nchunk);
  else if (e.R <= 8)
    k_ewald_gather<T, 8><<<gg, tb, 0, s>>>(e, n, w.frac, w.order, w.sp_of, c6, ci, tab, hsp, w.gpart, nchunk);
  else if (e.R <= 16)
    k_ewald_gather<T, 16><<<gg, tb, 0, s>>>(e, n, w.frac, w.order, w.sp_of, c6, ci, tab, hsp, w.gpart, nchunk);
  else
    k_ewald_gather<T, 32><<<gg, tb, 0, s>>>(e, n, w.frac, w.order, w.sp_of, c6, ci, tab, hsp, w.gpart, nchunk);
  FD3_LAUNCHED();
  const int ab = (n + tb - 1) / tb;
  k_ewald_finish<<<ab, tb, 0, s>>>(e, n, w.frac, w.order, w.sp_of, c6, dc6, ci, tab, w.gpart, nchunk, gcn, gpos,
                                   mcell_part);
  FD3_LAUNCHED();
  *n_mcell = mcell_part ? ab : 0;
  return FD3_OK;
}

template int launch_ewald<double>(const EwaldGeom&, int, const double*, double, const int32_t*, const double*,
                                  const double*, const CellInfo*, const GreenPair*, const Tables*, const EwaldWork&,
                                  bool, double*, double*, double*, int*, int*, cudaStream_t);
template int launch_ewald<float>(const EwaldGeom&, int, const double*, double, const int32_t*, const double*,
                                 const double*, const CellInfo*, const GreenPair*, const Tables*, const EwaldWork&,
                                 bool, double*, double*, double*, int*, int*, cudaStream_t);

}  // namespace fd3
