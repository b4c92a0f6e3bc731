// lbl_kernels.cuh -- device-side data structures and kernel launchers.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "lbl_plan.h"

namespace lbl {

constexpr int kSegMaxBlk = 48;  // panels a LINF4 segment may span

// Resident TAPE3 lines (device pointers).
struct DevLines {
  const double* vnu;   // centres, coupling records holding the previous line's
  const double* vraw;  // centres as given (coupling records: Y coefficient)
  const float *sp, *alfa, *epp, *hwhms, *tmpalf, *pshift;
  const int32_t *mol, *iflg;
  const int64_t* bs;  // panel starts, nblk+1
  int64_t n, nblk;
};

// Line-shape tables, 1-based, kNfmx+1 entries each (device pointers).
struct DevShapes {
  const double *f1, *f2, *f3, *fg, *xver;
  const double* r1p;  // F1, FG, XVER, 0 per table index (one 32-byte record)
  // FP32 copies for split precision: F1, FG, XVER, 0 per index (16 bytes), F2, F3
  const float4* r1p32;
  const float *f2_32, *f3_32;
};

// Continuum coefficient table (device pointers).
struct DevMtckd {
  const double *self, *forn, *texp;
  double v0, dv, ref_press, ref_temp;
  int64_t n;
};

// What k_near_lines leaves for the read-panel walk about one near-wing line
// of one layer, in one 32-byte record.
struct NearPre {
  double vnu;     // pressure-shifted centre
  double reach;   // HWF3*ALFV + VNU, against the read panel's VFT
  double speak;   // peak for the R4 test
  int32_t pf_fl;  // first panel whose R1 buffer holds the window << 2 | flags
                  // (bit 0: survives the panel-independent tests; bit 1: R4 test applies)
  int32_t wj;     // window of that panel << 16 | the line's R4 point in it
};

// One accepted near-wing line of one layer as the fused panel kernel reads
// it: the constants of CNVFNV's three sums (src/oprop.f90:1283-1351) and the
// line's windows on the three global grids.  Packed by k_near_out in file
// order, 96 bytes (a multiple of 16, so a run of records moves with one bulk
// copy).
struct NearRec {
  double zint, zslope, sppsp, s0, s2, s3, sg, sx;
  int32_t lo1, hi1, lo2, hi2, lo3, hi3;
  int32_t pc;   // convolution panel
  int32_t pad;
};
static_assert(sizeof(NearRec) == 96, "NearRec is 96 bytes");

// Work buffers of one batch of layers; offsets come from LayerDev.
struct Work {
  const LayerDev* L;     // nlay entries
  int32_t nlay;
  // per-panel
  const double* vft;
  const int32_t* win_of;
  int32_t* nseg;         // radiation segments per panel
  double* seg;           // [panel][kMaxSeg][3]: start, radvi, rdel
  // windows
  const WinDev* win;
  double* r4;
  // far-wing raw lines (slot = line index - far_lo)
  double *f_vnu, *f_sp, *f_alfa, *f_epp, *f_spp;
  int8_t *f_ok, *f_co2;
  // shrunk lines
  double *s_vnu, *s_sp, *s_alfa, *s_epp, *s_spp;
  int8_t* s_co2;
  int64_t* s_count;      // per layer
  int64_t* b9_start;     // per layer TAPE9 block starts (local shrunk index)
  double* b9_vnuhi;
  int64_t* b9_count;     // per layer number of TAPE9 blocks
  // LINF4 segmenting: per (layer, start panel) count tables and segments
  int32_t *c_raw, *c_out;  // [far panel][kSegMaxBlk]
  int32_t *seg_blk, *seg_nblk;
  int64_t* seg_out;
  int64_t* seg_count;    // per layer
  // near-wing lines (slot = line index - near_lo)
  double *n_zslope, *n_str;  // n_str: 5 per slot (F1,F2,F3,FG,VER)
  double* n_sppsp;
  NearPre* n_pre;  // k_near_lines -> k_near_walk, k_near_out
  int2* n_blk;     // per near-range TAPE3 panel: read panel (-1 past the end), stop line
  // accepted near-wing lines packed in file order (slot = rank within the layer)
  NearRec* n_rec;
  double* n_rvnu;    // their TAPE3 centres (ascending), for the panels' candidate search
  int32_t* n_boff;   // per near-range TAPE3 panel: accepted lines of the earlier panels
  int32_t* n_cnt;    // per layer: accepted lines
  int32_t* n_hw3;    // per layer: widest R3 half-window of an accepted line (R3 points)
  // grids
  double *r1, *r2, *r3;
  double* absrb;
  double* od;
  // diagnostics
  int32_t* status;       // device error flag (0 ok)
  unsigned long long* counters;  // [0] F4 line-point evals, [1] near point triples
};

void upload_voicon();

cudaError_t launch_far_scale(const Work& w, const DevLines& ln, int64_t max_far, cudaStream_t s);
cudaError_t launch_shrink(const Work& w, const int64_t* bs, const int64_t* blk_base,
                          int64_t nblk_total, cudaStream_t s);
// Far-wing variants the autotuner chooses among: 224, 352 or 480 adders per
// window CTA (3, 2 or 1 CTAs per SM).
constexpr int kFarVariants = 3;
cudaError_t launch_far_wing(const Work& w, int32_t nwin_total, const int32_t* win_order,
                            const int32_t* win_layer, int precision, int variant,
                            cudaStream_t s);
// Near-wing line scaling: per line and layer (k_near_lines), the read-panel
// walk per layer (k_near_walk: one warp, the layer's panel origins, window
// limits, current R4 and a ring of line records in shared memory), then
// the window limits of every line (k_near_out, per TAPE3 panel).
constexpr int kWalkRing = 4;  // TAPE3 panels of line records in flight
inline size_t near_walk_smem(int64_t npanel, int64_t nwin) {
  const size_t d = ((size_t)(npanel + nwin + kR4Stride) * sizeof(double) + 31) / 32 * 32;
  return d + (size_t)kWalkRing * 256 * sizeof(NearPre) + (size_t)(npanel + nwin) * sizeof(int32_t);
}
constexpr size_t kNearWalkSmemMax = 220 * 1024;
cudaError_t launch_near_lines(const Work& w, const DevLines& ln, int64_t max_near,
                              cudaStream_t s);
cudaError_t launch_near_walk(const Work& w, const DevLines& ln, int64_t max_panel,
                             int64_t max_win, int64_t max_nblk, cudaStream_t s);
cudaError_t launch_continuum(const Work& w, const DevMtckd& ck, double xself, double xfrgn,
                             double xrayl, double xco2c, double xo2cn, double xn2cn,
                             cudaStream_t s);
// RADFNI segments of every panel (needs only the plans).
cudaError_t launch_panel_segs(const Work& w, int64_t npanel_total, const int32_t* panel_layer,
                              const int64_t* panel_base, double* segs, int32_t* nseg,
                              cudaStream_t s);
// Every panel's candidate records (after k_near_out has packed the layers'
// accepted near-wing lines).
cudaError_t launch_panel_ranges(const Work& w, int64_t npanel_total, const int32_t* panel_layer,
                                const int64_t* panel_base, int64_t* rng, cudaStream_t s);
// Variants of the fused panel kernel the autotuner chooses among.
constexpr int kPanelVariants = 3;
int panel_stage_of(int variant);
cudaError_t launch_panels(const Work& w, const DevShapes& sh, int64_t npanel_total,
                          const int32_t* panel_layer, const int64_t* panel_base,
                          const int64_t* rng, const double* segs, const int32_t* nseg,
                          int precision, int variant, cudaStream_t s);
constexpr int kPanelSegMax = 48;  // RADFNI segments kept per panel (3 doubles each)
// One merge step (EMINIT when first) for the layer whose LayerDev is Ld.
cudaError_t launch_merge(const LayerDev* Ld, const double* vft_panel, const double* od,
                         int64_t npts, int first, double dv_old, int64_t n_old,
                         const double* rad_in, const double* tr_in, double* rad_out,
                         double* tr_out, double tbnd, double emis, int iemit, double tzu,
                         cudaStream_t s, int precision = LBL_PREC_FP64, int down = 0,
                         double tbnd_last = 0., double tzl_tangent = 0., double refl = 0.);
constexpr double kRADCN1 = 1.191042722E-12;  // src/phys_consts.f90:73
constexpr double kRADCN2 = 1.4387752;        // src/phys_consts.f90:74
// Temperatures of one EMIN step: XKT = T/RADCN2 and RADCN2/T for the layer
// and for its upper boundary (XKTA; zero when the boundary is absent).
struct EminT {
  double xkt, rk, xkta, rka;
};
__host__ __device__ inline EminT emin_temps(double tave, double tzu) {
  return {tave / kRADCN2, kRADCN2 / tave, tzu / kRADCN2, kRADCN2 / tzu};
}
// Consecutive layers on one grid merged in one pass: the first may be the
// bottom layer (EMINIT) or regrid the field below it (RADNN ITYPE>0); the
// rest share its grid, so the radiance and transmittance stay in registers
// from layer to layer and each layer's optical depth is read once.
constexpr int kMergeRunMax = 32;
struct MergeRun {
  int32_t nl;                    // layers in this launch (1..kMergeRunMax)
  int32_t first;                 // the launch starts at the bottom layer
  int32_t itype;                 // regrid of the incoming field (0: same grid)
  int32_t n_old;                 // points of the incoming field
  int32_t down;                  // looking up (IPATHL=3): RADNN IPATH=3
  int32_t tangent;               // the symmetric tangent path (IPATHL=2):
                                 // each layer crossed twice, RADNN IPATH=2
  double tbnd_last;              // > 0: the boundary beyond the run's last layer
                                 // (EMBND, the profile's last layer looking up)
  int64_t od_off[kMergeRunMax];  // each layer's optical depths in Work::od
  EminT t[kMergeRunMax];
  // the reflected atmosphere (IPATHL=-1, specular): the boundary
  // reflectivity BNDRFL(1); 0 otherwise
  double refl;
  // tangent path and reflected atmosphere: XKTB (the lower level's
  // temperature / RADCN2) and its reciprocal RADCN2 / TZL, per layer (0 when
  // TZL <= 0)
  double tb_xkt[kMergeRunMax], tb_rk[kMergeRunMax];
};
// Points [f_lo, f_hi) of the run's grid (f_hi < 0: to the end).
cudaError_t launch_merge_run(const MergeRun& m, const double* vft_panel, const double* od,
                             int64_t npts, double dv, const double* rad_in, const double* tr_in,
                             double* rad_out, double* tr_out, double tbnd, double emis, int iemit,
                             cudaStream_t s, int precision, int64_t f_lo = 0, int64_t f_hi = -1);
// Radiance Jacobians: one layer's forward merge plus its derivative rows,
// the carrying of lower layers' rows through one merge step, the top
// segment's transmittance products, and a central difference.
cudaError_t launch_jac_layer(const LayerDev* Ld, const double* vft_panel, const double* od,
                             int64_t npts, int first, double dv_old, int64_t n_old,
                             const double* rad_in, const double* tr_in, double* rad_out,
                             double* tr_out, double tbnd, double emis, double tzu,
                             double* const* d, const double* const* dtau, int np,
                             int mode, int k0, cudaStream_t s);
cudaError_t launch_jac_prop(const LayerDev* Ld, const double* od, int64_t npts, double dv_old,
                            int64_t n_old, const double* in, double* out, int64_t stride,
                            int nrows, cudaStream_t s);
cudaError_t launch_jac_top(const double* od, const int64_t* od_off, int nlay, int a, int np,
                           int64_t n, double* rows, const double* low, cudaStream_t s);
cudaError_t launch_jac_diff(double* plus, const double* minus, int64_t n, double rh,
                            cudaStream_t s);
// Means of nrows rows (n points each) over channels [cb[c], cb[c+1]).
cudaError_t launch_chan_mean(const double* x, int64_t n, int nrows, const int64_t* cb,
                             int64_t nchan, double* out, cudaStream_t s);
constexpr int kJacMaxParams = 8;
// SCANFN: SHRKSC's compression of spec (n points, groups of ir, 1 - x when
// jabs) into sc (n / ir points), then CONVSC's sums on the global output
// grid, one thread per output point (the inputs ilo..ihi, 1-based).
// SCNINT/INTERP: the chunks of a host replay (lbl_plan.h ScnChunk, same
// layout), the weights C1..C4 (4 x 203), out of the replay's size.
struct ScnChunkDev {
  int64_t out0, panel, i0;
  double p0;
  int32_t count, zero;
};
cudaError_t launch_scnint(const ScnChunkDev* chunks, int64_t nchunk, const double* spec,
                          int64_t n, const double* coef, double vratio, double* out,
                          cudaStream_t s);
// CNVRCT / CNVVRC / CNVVRL (mode 0 / 5 / 6): weighted means of the input
// over boxes at v1 + j*dvo (j < n_out; every box inside the input): half
// width hwhm (mode 0) or widths set by the field-of-view half angle bfov.
cudaError_t launch_scan_rect(const double* spec, int64_t n, int jabs, int mode, double v1,
                             double dvo, double hwhm, double bfov, double v1i, double dvi,
                             double* out, int64_t n_out, cudaStream_t s);
cudaError_t launch_scan(const double* spec, int64_t n, int ir, int jabs, double* sc, int64_t ilo,
                        int64_t ihi, double zint, double ratio, double zbound, double zslope,
                        double xnorm, const double* xf, int64_t nfmax, double* out,
                        int64_t n_out, cudaStream_t s);
// PNLINT re-grid of one layer (one CTA per segment of the host plan);
// a: the 4 x 101 Lagrange weights.
cudaError_t launch_pnlint(const PnlSeg* seg, int64_t nseg, const double* a, const double* od,
                          int64_t n_in, double ratdv, double* out, int64_t n_out,
                          cudaStream_t s);

void init_kernel_attributes();

}  // namespace lbl
