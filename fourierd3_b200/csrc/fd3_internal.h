// Internal declarations shared by the .cu files of libfd3 (not part of the ABI).
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include "fd3_common.cuh"

namespace fd3 {

// ---- error plumbing ---------------------------------------------------------
void set_error(const char* where, const char* what);
void count_launch();
#define FD3_CUDA(call)                                            \
  do {                                                            \
    cudaError_t e_ = (call);                                      \
    if (e_ != cudaSuccess) {                                      \
      ::fd3::set_error(#call, cudaGetErrorString(e_));            \
      return FD3_ECUDA;                                           \
    }                                                             \
  } while (0)
#define FD3_LAUNCHED()                                            \
  do {                                                            \
    ::fd3::count_launch();                                        \
    cudaError_t e_ = cudaGetLastError();                          \
    if (e_ != cudaSuccess) {                                      \
      ::fd3::set_error("kernel launch", cudaGetErrorString(e_));  \
      return FD3_ECUDA;                                           \
    }                                                             \
  } while (0)

// ---- cell list geometry ------------------------------------------------------
struct CellGrid {
  int nb[3];        // bins per axis
  int reach[3];     // bins to visit on each side
  double cell[9];   // Angstrom rows
  double inv[9];    // Angstrom inverse (host-computed; only used for binning)
  double rc2;       // r_cut^2 (Angstrom^2) for the exact predicate
  double r_cut;
};
int make_cell_grid(const double* h_cell, double r_cut, CellGrid* g);

// Device arrays of a built cell list (all sized from the plan workspace).
struct CellList {
  int* bin_of;      // [N]   bin id of each atom
  int* bin_count;   // [K]   histogram (zeroed before use)
  int* bin_start;   // [K+1] exclusive scan
  int* order;       // [N]   atom ids sorted by bin, then by id
  double4* xs;      // [N]   bin-sorted positions (A) + species in .w
  int4* meta;       // [N]   bin-sorted {off_x, off_y, off_z, atom id}
  int4* off;        // [N]   per atom {off_x, off_y, off_z, bin}
};

// counting sort of keys[N] in [0, K): out order sorted by key then by index.
// counts[K] and starts[K+1] are workspace; counts must be zeroed by the caller.
int counting_sort(const int* keys, int n, int K, int* counts, int* starts, int* order, cudaStream_t s);
int scan_exclusive(const int* in, int n, int* out, cudaStream_t s);   // out[n] = total

int build_cell_list(const CellGrid& g, int n, const double* pos_ang, const int32_t* species, CellList& cl,
                    cudaStream_t s);

// Per-atom records of the CN pairs (neighbour, and {f'(r)/r, Bohr vector} as one 4-wide record),
// written by the CN kernel and streamed by its adjoint; ad is double4 (plain form) or float4
// (mixed form).
struct HitStore {
  int* j;
  void* ad;
  int* n;
  int* ovf;     // count of bins / atoms that need the global-memory fallback (zeroed per call)
  int cap;
  bool is_double;
};
constexpr int kHitCap = 160;

// fused CN + C6 factors over the cell list (one CTA per bin)
int launch_cn_c6_cells(const CellGrid& g, int n, const CellList& cl, const double* pos_ang,
                       const int32_t* species, const Tables* tab, const double* eigvecs, int R, double* cn,
                       double* c6, double* dc6, double* self_part, int* n_self_blocks, const HitStore& hs,
                       cudaStream_t s);
// CN adjoint: grad = out_scale * (grad + dE/dx_CN) (Hartree/Bohr in); virial partials (9 per block)
int launch_cn_adjoint_cells(const CellGrid& g, int n, const CellList& cl, const double* pos_ang,
                            const int32_t* species, const Tables* tab, const double* gcn, double* grad,
                            double out_scale, double* vir_part, int* n_blocks, const HitStore& hs,
                            cudaStream_t s);

// direct pairwise lattice sum (float64 accuracy oracle on the device)
int launch_direct_pairs(const CellGrid& g, int n, const CellList& cl, const double* c6, const Tables* tab, int R,
                        int S, const GreenPair* gp, double* dEdc, double* grad, double* part, int* n_blocks,
                        cudaStream_t s);
size_t direct_scratch_doubles(int S, int R);
int launch_direct_tail_gcn(int n, const int32_t* species, const double* c6, const double* dc6, const double* dEdc,
                           const Tables* tab, const GreenPair* gp, int S, int R, double rc_bohr, const CellInfo* ci,
                           double* sp_part, int sp_blocks, double* A, double* tail, double* T, double* gcn,
                           cudaStream_t s);
int launch_direct_finalize(const double* pair_part, int n_pair, const double* tail, const double* cnv_part, int n_cnv,
                           const CellInfo* ci, double* energy, double* stress, cudaStream_t s);

// edge-list CN path
// Edges sorted by source and by destination (stable counting sorts of the edge ids): the
// per-atom segments the fixed-order CN sum and its adjoint walk.
struct EdgeIndex {
  int *ks, *kd;         // [E] source / destination keys
  int *ord_s, *ord_d;   // [E] edge ids by source / by destination
  int* cnt;             // [N] counting-sort scratch
  int *st_s, *st_d;     // [N+1] segment starts
  int* bad;             // [1] set when an edge index is outside 0..N-1
};
int launch_edge_index(int64_t n_edges, int n, const int64_t* src, const int64_t* dst, const EdgeIndex& ei,
                      cudaStream_t s);
// edges with |r|^2 >= mask_r2 (Bohr^2) contribute nothing; +inf: every edge counts
int launch_cn_edges_seg(int64_t n_edges, int n, const double* pos, const int32_t* species, const int64_t* src,
                        const int64_t* dst, const double* shift, const Tables* tab, double mask_r2,
                        const EdgeIndex& ei, double* cn, cudaStream_t s);
int launch_cn_adjoint_edges_seg(int64_t n_edges, int n, const double* pos, const int32_t* species,
                                const int64_t* src, const int64_t* dst, const double* shift, const Tables* tab,
                                double mask_r2, const double* gcn, const EdgeIndex& ei, double* gpos,
                                double* gshift, cudaStream_t s);
int launch_c6_atoms(int n, const int32_t* species, const Tables* tab, const double* eigvecs, int R,
                    const double* cn, double* c6, double* dc6, double* self_part, int* n_self_blocks,
                    cudaStream_t s);

// neighbour export
int launch_nbr_count(const CellGrid& g, int n, const CellList& cl, const double* pos_ang, int* counts,
                     cudaStream_t s);
int launch_nbr_fill(const CellGrid& g, int n, const CellList& cl, const double* pos_ang, const int* row_start,
                    int64_t* src, int64_t* dst, int32_t* shift, cudaStream_t s);

// ---- mesh ---------------------------------------------------------------------
struct MeshGeom {
  int n[3];       // mesh points per axis
  int nzh;        // nz/2 + 1
  int t[3];       // tile edge per axis (divides n)
  int nt[3];      // tiles per axis
  int ns[3];      // source tiles per axis that can reach a tile
  int order;      // p
  int lagrange;   // 0: B-spline (spme), 1: Lagrange (pme)
  int S, R;
  int filter_kt;  // filter k-tile width (0: register kernel), -1: default for (S, R)
  int spread_zc;  // z-tiles per column chunk of the spread (0: per-tile kernel), -1: default
  int spread_cap; // staged atoms per column chunk at most (0: as many as shared memory holds)
  int fft_x;      // fused x-pass (2D cuFFT + x FFT/filter kernel): 1 on, 0 off, -1 default
  int xpencil;    // kz values per pencil of the fused x-pass (1, 2, 4), -1 default
  int xq;         // TMA x-pass: q values per unit (4, 8, 16, 32), -1 default
  int xranks;     // TMA x-pass: ranks per unit (1, 2, 4), -1 default
  int filter_mma; // float spectrum: 1 tensor-core (tcgen05) filter where it applies, 0 CUDA cores, -1 default
  int gather_tile; // fused-path gather: 1 tile-staged TMA gather where it applies, 0 or -1 (default) per-atom
  int fft_yz;      // float mesh, 2D-transform paths: fused (y, z) cluster kernels (1 pairs, 2 quad forward), 0 cuFFT, -1 default (1)
  int qpitch;      // complex values per ky row of the half spectrum: nzh, or nzh + 1 (16-byte rows) when the
                   // TMA x-pass and the fused (y, z) transforms share it; 0 = nzh
  const float* win_axes;  // SPME, mixed form: sinc(m/n)^(2p) per axis, [nx | ny | nz/2+1] (null: none)
};
// h_expect (optional, host, copied into the launch): the cell the caller's host-side geometry (cell
// list bins) was built from; a device cell that differs sets ci->stale
int launch_cellinfo(const double* cell, double scale, CellInfo* ci, cudaStream_t s,
                    const double* h_expect = nullptr);
// energy, forces [n*3] and stress [9] made NaN when ci->stale is set
int launch_poison_if_stale(const CellInfo* ci, int n, double* energy, double* forces, double* stress,
                           cudaStream_t s);
int launch_mesh_keys(const MeshGeom& mg, int n, const double* pos, double pos_scale, const int32_t* species,
                     const CellInfo* ci, int* keys, cudaStream_t s);
// Per-atom stencil records in (tile, species)-sorted order, written by the spread launcher and
// read again by the gather (T = mesh precision).
struct MeshRecords {
  int4* b;      // [N] {base_x, base_y, base_z, species}
  void* w;      // [N][3][P] weights
  void* dw;     // [N][3][P] d weight / d local coordinate
  void* c;      // [N][R] rank factors
};
// Fused (y, z) plane transforms of the float mesh (ny = nz = 256; planes = nchannels x nx, the
// layouts of the batched 2D cuFFT R2C / C2R they replace).
bool yzfft_applies(const MeshGeom& mg);
// variant 1: clusters of 2 CTAs (one per SM); 2: the forward on clusters of 4 (two per SM), the
// inverse on pairs.
int launch_yz_forward(const MeshGeom& mg, int nchannels, int variant, const float* rho, void* spec,
                      cudaStream_t s);
int launch_yz_inverse(const MeshGeom& mg, int nchannels, int variant, const void* spec, float* rho,
                      cudaStream_t s);
// Whether the tile-staged (TMA) gather applies to this mesh for elements of `elem` bytes.
bool gather_tile_applies(const MeshGeom& mg, size_t elem);
// records: 0 = write the stencil records (with the rank factors) and spread; 1 = the records'
// nodes and weights are written already (kSpreadRecordsOnly on another stream): write the rank
// factors and spread; 2 (kSpreadRecordsOnly) = write the records' nodes and weights only (they
// need the positions and the mesh sort, not C6).
constexpr int kSpreadRecordsOnly = 2;
template <typename T>
int launch_spread(const MeshGeom& mg, int n, const double* pos, double pos_scale, const int32_t* species,
                  const double* c6, const CellInfo* ci, const int* key_start, const int* order,
                  const MeshRecords& rec, T* rho, cudaStream_t s, int records = 0);
template <typename T>
int launch_filter(const MeshGeom& mg, const CellInfo* ci, const GreenPair* gp, const GreenPairF* gpf,
                  const float4* gtab, const Tables* tab, const float* deconv, int spme, void* spec, double* part,
                  int* n_blocks, cudaStream_t s);
// fused x-pass: forward x FFT + filter + inverse x FFT on the (y, z)-transformed spectrum
template <typename T>
int launch_xfilter(const MeshGeom& mg, const CellInfo* ci, const GreenPair* gp, const GreenPairF* gpf,
                   const float4* gtab, const Tables* tab, const float* deconv, int spme, void* spec, double* part,
                   int* n_blocks, cudaStream_t s);
// kz width of the fused x-pass pencils for this mesh (0: the fused path does not apply)
int xfilter_pencil(const MeshGeom& mg, int is_double);
// TMA fused x-pass (float spectrum): units of Q flattened (y, kz) values x all x x RG ranks x S
bool xpass_applies(const MeshGeom& mg, int Q, int RG);
int launch_xpass(const MeshGeom& mg, int Q, int RG, const CellInfo* ci, const GreenPairF* gpf, const float4* gtab,
                 const Tables* tab, const float* deconv, int spme, void* spec, double* part, int* n_blocks,
                 cudaStream_t s);
// tensor-core filter (float spectrum, tcgen05 kind::tf32, at most 64 species and 8 ranks)
bool filter_mma_applies(const MeshGeom& mg);
bool filter_mma_on(const MeshGeom& mg);
int launch_filter_mma(const MeshGeom& mg, const CellInfo* ci, const float4* gtab, const Tables* tab,
                      const float* deconv, int spme, void* spec, double* part, int* n_blocks, cudaStream_t s);
// mixed form: per-call table of G and its k-derivatives per species pair (gtab of the filter)
int launch_green_table(const MeshGeom& mg, const CellInfo* ci, const GreenPair* gp, const Tables* tab, void* table,
                       cudaStream_t s);
size_t green_table_bytes(int S);
int filter_max_blocks();
int filter_default_kt(int S, int R, size_t tsize);
int spread_chunk_in_effect(const MeshGeom& mg, size_t tsize);
bool filter_kt_valid(int kt, int S, int R, size_t tsize);
template <typename T>
int launch_gather(const MeshGeom& mg, int n, const double* pos, double pos_scale, const int32_t* species,
                  const double* c6, const double* dc6, const CellInfo* ci, const Tables* tab, const int* order,
                  const int* key_start, const MeshRecords& rec, const T* phi, double* gcn, double* gpos,
                  double* mcell_part, int* n_blocks, cudaStream_t s);

// ---- D4 coordination numbers in k-space (cnfunc = 'd4') ----------------------------------
// Per species pair of the erfc CN function (pair_pot.py:286-325): r0 = rcov_cn_A + rcov_cn_B,
// delta = k1 exp(-(|EN_A - EN_B| + k2)^2 / k3), Taylor constants c0, c2 of the small-k branch.
struct CnPair {
  double r0, delta, c0, c2;
};
constexpr double kCn4K0 = 7.5, kCn4K1 = 4.10451, kCn4K2 = 19.08857, kCn4K3 = 2.0 * 11.28174 * 11.28174;
constexpr int kCn4MaxSpecies = 8;
int cn4_gather_blocks(int n);
int launch_cn4_values(int n, int adjoint, const double* gcn, const CellInfo* ci, double* vals, cudaStream_t s);
// forward (adjoint = 0): out = G rhat; adjoint: k-space strain partials (9 per block) and out <- G out
template <typename T>
int launch_cn4_filter(const MeshGeom& mg, int adjoint, const CellInfo* ci, const CnPair* cp, const float* deconv,
                      int spme, const void* rhat, void* out, double* part, int* n_blocks, cudaStream_t s);
// mode 0: CN values from phi; mode 1: gradient gather (phi, psi), volume strain partials, cell partials
template <typename T>
int launch_cn4_gather(const MeshGeom& mg, int n, int mode, const double* pos, double ps, const CellInfo* ci,
                      const int* order, const MeshRecords& rec, const void* phi, const void* psi,
                      const double* cnself, const double* gcn, double* cn, double* gpos, double out_scale,
                      double* vir_part, double* mcell_part, cudaStream_t s);

// ---- direct Ewald k-sum --------------------------------------------------------------
struct EwaldGeom {
  int ns[3];   // Miller-index box (fftfreq order per axis)
  int S, R;
};
struct EwaldWork {
  int* keys;      // [N]
  int* counts;    // [S]
  int* sp_start;  // [S+1]
  int* order;     // [N] atoms sorted by species
  int4* sp_of;    // [N] species of each sorted slot
  double* frac;   // [N*3] fractional coordinates, sorted order
  void* spec;     // [S*R*nk] structure factors
  void* hspec;    // [S*R*nk] H = G S
  double* kpart;  // filter partials
  double* gpart;  // [N * nchunk * (R+3)] gather partials
};
int ewald_chunks(int nk);
template <typename T>
int launch_ewald(const EwaldGeom& eg, int n, const double* pos, double ps, const int32_t* species,
                 const double* c6, const double* dc6, const CellInfo* ci, const GreenPair* gp, const Tables* tab,
                 const EwaldWork& w, bool need_grad, double* gcn, double* gpos, double* mcell_part, int* n_kspc,
                 int* n_mcell, cudaStream_t s);

// ---- finalisation ---------------------------------------------------------------
struct Partials {
  const double* self;  int n_self;     // 1 value per block
  const double* kspc;  int n_kspc;     // 7 per block: q, V00 V11 V22 V01 V02 V12
  const double* cnv;   int n_cnv;      // 9 per block (CN virial), may be 0
  const double* mcell; int n_mcell;    // 9 per block: sum_i s_iA g_ia, may be 0
};
int launch_finalize(const Partials& p, const CellInfo* ci, int mode, double e_scale, double* energy,
                    double* out9, cudaStream_t s);

}  // namespace fd3
