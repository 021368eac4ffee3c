// kernels.cuh -- launcher declarations shared by the kernel and host files.
#pragma once
#include <vector>

#include "common.cuh"

namespace blgpu {

// metric tables in the storage precision T (1-based, see Axis)
template <typename T> struct MetT {
  const T *xF, *xC, *xrF, *xrC;
  const T *yF, *yC, *yrF, *yrC;
  const T *zF, *zC, *zrF, *zrC;
  const T *w0, *w1;
  T nu, dpdx, dpdz;
};

// Launch shapes of the main kernels.  0 selects the built-in choice; the
// autotuner (blgpu_autotune) searches these per box.
struct Tiles {
  int rhs_kc;   // k-planes walked by one CTA of the RHS kernel (0: 8; TMA-fed 16 in FP32, 32 in FP64; FP32 two points 8, one 32)
  int rhs_by;   // RHS block is 32 x rhs_by threads (0: 8)
  int dct_nw;   // complex lines (warps) per CTA of the forward DCT, up to 16 in FP32 (8 two-pass) and 8 in FP64 (0: built-in)
  int dftz_rk;  // z wavenumbers per warp in the z-DFT, 4 or 8 (0: 8)
  int proj_by;  // projection block is 32 x proj_by threads (0: 4)
  int zdft;     // mixed-form z transforms: 1 FP32 sums, 2 mma.sync TF32, 3 tcgen05 (0: tcgen05, else mma.sync, else sums)
  int rhs_pts;  // FP32 DNS RHS: 1 one point per thread, 2 two points, 3 two points packed in FP32x2
                // instructions, 4 the same fed by TMA (0: 4 where its tensor maps exist, else 2);
                // FP64 DNS: 1 one point with global loads, 4 one point TMA-fed, 0 or 2 two points
  int thomas;   // y-solve: 1 register ring, 2 TMA tiles where the box allows (one thread per mode), 3 the
                // tiles with each mode's rows split over 16 threads (0: 3 where the tiles exist, else 1)
  int idct_nw;  // complex lines (warps) per CTA of the inverse DCT, as dct_nw (0: built-in)
  int xfft;     // x transforms: 1 Stockham, 2 two-pass registers (0: two-pass where built for N; FP64: N = 812)
};

// boundary data (FP64, 1-based like the Fortran vectors)
struct BcData {
  const double *U_inlet, *V_inlet, *W_inlet;  // (nyg) (ny) (nyg)
  const double *U_top, *V_top, *W_top;        // (nx) (nxg) (nxg)
  int n_modes, m_modes;
  const double *zmode, *tmode;                // (n) (m)
  const double2 *qu, *qv, *qw;                // (nyg|ny, n, m) complex
  const double *ut, *vt, *wt;                 // optional precomputed inflow perturbation planes
  int lund;                                   // 0 modes, 3 Lund plane, 5 Lund fluctuations
  const double *lu, *lv, *lw;                 // Lund planes (nyg,nzg) (ny,nzg) (nyg,nz), j fastest
  const double *wm_ax, *wm_az;                // wall model: tau/nu_wall at (i,k), i=2..nx-1, k=2..nzg-2 (or null)
};

// Lund recycling/rescaling inflow state (rescaled_inlet_bc.f90:60-345), FP64.
// inst and mean hold four profiles back to back: U at the recycling station
// (nyg), U at the inlet (nyg), V at the station (ny), V at the inlet (ny);
// inst has one more entry, the z-mean of 0.5(U(1)+U(2))V(1) at the station.
// The four interpolation maps are m = 0 (U/W rows, wall units), 1 (U/W rows,
// delta units), 2 (V rows, wall units), 3 (V rows, delta units), each with
// nyg slots: rowi = -1 row 1 (left 0), 0 top value, j > 1 the pair (j-1, j).
struct LundData {
  int mode, ir;
  double delta_inlet, T_resc;
  double *inst, *mean;
  double *rowc, *wgt, *mprof;  // rowc 4 x nyg; wgt: Weig (nyg) + Wei (ny); mprof: U inner/outer, V inner/outer
  int *rowi, *err;
  double *lu, *lv, *lw, *diag;  // diag: Uinf, delta_resc, delta_inlet, theta_resc, theta_inlet,
                                //       utau_resc, utau_inlet, gamma
};

// ---- stencil.cu ----
struct RhsMaps {  // CUtensorMap bytes of the planes of U, V, W of one FP32 buffer set (TMA-fed RHS):
  alignas(64) unsigned char f[3][128];  // neighbourhood tiles (72 x 10)
  alignas(64) unsigned char p[3][128];  // point-wise tiles (64 x 8)
};
// false when a map cannot be encoded (the RHS then uses the kernels with
// global loads)
bool rhs_maps(const Geo &g, const float *U, const float *V, const float *W, RhsMaps *out);
bool rhs_maps64(const Geo &g, const double *U, const double *V, const double *W, RhsMaps *out);
// mi, mo, mf: tensor maps of the buffers of U V W, Uo Vo Wo and F1 (the
// TMA-fed DNS kernels: FP32 with rhs_pts 0 or 4, FP64 unless rhs_pts 1), or null; err: device flag, bit 64 set when a plane
// copy missed its wait limit; wait_limit: mbarrier polls before giving up
// (< 0: the built-in limit)
template <typename T>
void launch_rhs_rk(const Geo &g, const MetT<T> &m, int mode, bool les, const T *U, const T *V, const T *W,
                   const T *nut, const T *Uo, const T *Vo, const T *Wo, T *F1u, T *F1v, T *F1w, T *Un, T *Vn, T *Wn,
                   const Scalars *sc, double c1, double c2, const Tiles &tl, const RhsMaps *mi, const RhsMaps *mo,
                   const RhsMaps *mf, int *err, int wait_limit, cudaStream_t st);
template <typename T>
void launch_project(const Geo &g, const MetT<T> &m, const T *p, const double *p0, const float *p0g, T *U, T *V,
                    T *W, T *P,
                    const Scalars *sc, int save_p, const Tiles &tl, cudaStream_t st);
int bc_x_parts(const Geo &g);
template <typename T>
void launch_bc(const Geo &g, const BcData &bc, T *U, T *V, T *W, const T *Uo, const T *Vo, const T *Wo,
               Scalars *sc, double rkt, double *qx_part, double qy, double length_y, cudaStream_t st);
// save_time: the reduction's last block also saves the step's start time
// (sc->to = sc->t, what launch_set_time phase 0 does)
template <typename T>
void launch_dt(const Geo &g, const T *U, const T *V, const T *W, Scalars *sc, double cfl, double dtvis,
               bool save_time, cudaStream_t st);
void launch_set_time(Scalars *sc, int phase, double coef, cudaStream_t st);
template <typename T>
void launch_maxdiv(const Geo &g, const T *U, const T *V, const T *W, unsigned long long *out, cudaStream_t st);

template <typename T>
void launch_smagorinsky(const Geo &g, const T *U, const T *V, const T *W, const double *cs2, T *nut, cudaStream_t st);
// dynamic Smagorinsky (LES = 2 z-averaged, 3 pointwise), FP64 on dense work arrays;
// returns the number of kernels launched
size_t dyn_smagorinsky_work_bytes(int nxg, int nyg, int nzg);
template <typename T>
int launch_dyn_smagorinsky(const Geo &g, const T *U, const T *V, const T *W, double *work, int model, T *nut,
                           cudaStream_t st);
template <typename T>
void launch_stats(const Geo &g, const T *U, const T *V, const T *W, const T *P, const T *nut, double *out,
                  cudaStream_t st);
template <typename T>
void launch_law_of_wall(const Geo &g, const T *U, double *utau, int *iters, int jref, cudaStream_t st);
template <typename T>
void launch_lund(const Geo &g, const LundData &L, const T *U, const T *V, const T *W, const Scalars *sc, int phase,
                 cudaStream_t st);
// dir 0: host-layout FP64 stage -> box (bit 32 of *flag set on a NaN or infinity; flag may be null);
// dir 1: box -> stage
template <typename T>
void launch_repack(const Geo &g, int dir, double *stage, T *box, int n1, int n2, int n3, int *flag, cudaStream_t st);

// ---- spectral.cu ----
// Transform plan of one axis length n (device tables)
template <typename T> struct FftPlan {
  int n;
  int nst;            // number of stages
  int rad[24];        // radices, applied in order
  const typename vec2<T>::type *tw;    // W_n^t = exp(-2 pi i t / n), t = 0..n-1
  const typename vec2<T>::type *post;  // exp(-i pi k / (2n)), k = 0..n-1 (DCT twiddle)
};

struct Spec {  // spectral layout of the Poisson solve
  int N;      // nxp = nx-2 (DCT length)
  int M;      // nzp = nz-2 (DFT length)
  int NM;     // nm  = ny-1 (unknowns per mode)
  int MH;     // M/2 + 1 (stored z wavenumbers)
  int rx;     // row pitch of the spectral arrays (>= N, multiple of 32)
};

template <typename T>
void launch_div_dct(const Geo &g, const Spec &s, const FftPlan<T> &pl, const T *U, const T *V, const T *W, T *R,
                    int nw, int xfft, cudaStream_t st);
template <typename T>
void launch_dft_z(const Spec &s, const T *R, typename vec2<T>::type *C, const typename vec2<T>::type *ztab, int inverse,
                  int rk, cudaStream_t st);
// FP64 z transforms on the FP64 tensor-core MMA (8 <= M <= 254): the host
// tables (cos, then sin, [rows][Kp] each) and the forward / inverse launch
void zdft64_tables(const Spec &s, std::vector<double> &t);
void launch_zdft64(const Spec &s, double *R, double2 *C, const double *tab, int inverse, cudaStream_t st);
// H0 (mixed form): the kz = 0 modes kx < klow are solved in FP64 into
// H0[NM][klow] and zeroed in C; null for the FP64 form
template <typename T>
void launch_thomas(const Spec &s, typename vec2<T>::type *C, const double *piv, const double *dl, const double *du,
                   double *H0, int klow, cudaStream_t st);
// p0[NM][N] = inverse cosine sum of H0 (cm[kx][i] = w_kx cos(pi kx (2i+1)/2N)/(N M))
// and grad = FP32 x and y differences of p0 ([2][NM][N])
void launch_kz0_idct(const Spec &s, const double *H0, int klow, const double *cm, double *p0, float *grad,
                     cudaStream_t st);
// ---- zdft_tc.cu: mixed-form z transforms on the tensor cores ----
// order of the square products (M/2+1 rounded up to 16) when served, else 0
int zdft_tc_qp(const Spec &s);
size_t zdft_tc_frag_words(const Spec &s);
void zdft_tc_fragments(const Spec &s, std::vector<uint32_t> &out);
// ---- zdft_umma.cu: the same transforms on tcgen05 tensor cores (TMEM) ----
int zdft_umma_qp(const Spec &s);
void zdft_umma_tables(const Spec &s, std::vector<uint32_t> &out);
struct ZdftMaps;
bool zdft_umma_maps(const Spec &s, float *R, float2 *C, ZdftMaps *out);
// err: device flag, bit 8 set when a copy or a product missed its wait limit
void launch_zdft_umma(const Spec &s, const ZdftMaps &maps, float *R, float2 *C, const uint32_t *tab, int inverse,
                      int nsm, int *err, cudaStream_t st);
// TMA tensor maps of R and C (CUtensorMap bytes) for the loads, and the
// 128-byte-swizzled ones the tcgen05 form stores through; false when unavailable
struct ZdftMaps {
  alignas(64) unsigned char r[128];
  alignas(64) unsigned char c[128];
  alignas(64) unsigned char rs[128];
  alignas(64) unsigned char cs[128];
};
bool zdft_tc_maps(const Spec &s, float *R, float2 *C, ZdftMaps *out);
// inverse = 0: R -> C (forward); 1: C -> R; nsm: persistent CTAs; err: device
// flag, bit 2 set when a TMA copy did not complete within the wait limit
void launch_zdft_tc(const Spec &s, const ZdftMaps &maps, float *R, float2 *C, const uint32_t *frag, int inverse,
                    int nsm, int *err, cudaStream_t st);
// ---- cufft_path.cu: the cuFFT comparison path (solve_poisson_gpu with cuFFT plans) ----
struct CufftPath;
// plans (set to stream st) and the 2N plane / mode arrays; 0 or -1 with msg
int cufft_path_create(const Spec &s, bool fp64, cudaStream_t st, CufftPath **out, char *msg, size_t cap);
void cufft_path_destroy(CufftPath *c);
size_t cufft_path_bytes(const CufftPath *c);
// divergence + symmetric pack + 2D forward transform; returns the cufftResult
template <typename T>
int cufft_path_forward(CufftPath *c, const Geo &g, const Spec &s, const T *U, const T *V, const T *W, cudaStream_t st);
// twiddle extract + y-solve (post = the DCT twiddles exp(-i pi i/2N) in T)
template <typename T>
void cufft_path_extract_solve(CufftPath *c, const Spec &s, const void *post, const double *piv, const double *dl,
                              const double *du, double *H0, int klow, cudaStream_t st);
template <typename T> int cufft_path_inverse_z(CufftPath *c);
// untwiddle + Hermitian extension + inverse x transform + rhs_p into the box
template <typename T>
int cufft_path_inverse_x(CufftPath *c, const Geo &g, const Spec &s, const void *post, T *p, cudaStream_t st);
// ---- thomas_tma.cu: the y-solve as one TMA-fed pass over tiles ----
struct ThomasMaps {  // CUtensorMap bytes of C and of the pivots
  alignas(64) unsigned char c[128];
  alignas(64) unsigned char p[128];
};
// false when the maps cannot be encoded or NM > 256 (the register-ring
// k_thomas then serves the box)
template <typename T>
bool thomas_maps(const Spec &s, void *C, double *piv, ThomasMaps *out);
// err: device flag, bit 4 set when a tile copy missed its wait limit;
// wait_limit: mbarrier polls before giving up (< 0: the built-in limit);
// scan: each mode's rows split over 16 threads (k_thomas_tile_scan)
template <typename T>
void launch_thomas_tile(const Spec &s, const ThomasMaps &maps, const double *dl, const double *du, double *H0,
                        int klow, int *err, int wait_limit, bool scan, cudaStream_t st);
// inverse pivots piv[b][kz][kx] of the y-solve (grid only; once per grid)
void launch_thomas_factors(const Spec &s, double *piv, const double *dd, const double *dl, const double *du,
                           const double *kxx, const double *kzz, cudaStream_t st);
template <typename T>
// err: device flag, bit 16 set when a row copy of the two-pass kernel missed its wait limit
void launch_idct(const Geo &g, const Spec &s, const FftPlan<T> &pl, const T *R, T *p, int nw, int xfft, int *err,
                 cudaStream_t st);
// shared memory of a DCT CTA of `lines` warps; split: that of xfft_split, 0 for the Stockham kernels
size_t dct_smem_bytes(int n, int elem_bytes, int lines, int split);
// the split A of N = A B served by the two-pass FP32 x transforms, 0 if none
int xfft_split(int n);
// the R-point DFT constants of the odd register butterflies (once per device)
int upload_dft_constants();
int dct_lines_per_cta(int n, int elem_bytes, bool inverse, int split);
int dct_max_lines(int elem_bytes, int split);  // launch bound of the DCT kernels, in warps

}  // namespace blgpu
