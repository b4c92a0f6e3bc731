// lbl_plan.h -- per-layer plan shared by the host planner and the kernels.
//
// The reference streams each layer through 2400-point panels (PANEL,
// src/oprop.f90:1371) and 2500-point far-wing windows (LBLF4,
// src/oprop.f90:3641).  Here the whole layer lives in device memory on
// three global grids (spacing DV, 4*DV, 16*DV, indexed from the panel-0
// origin VFT0 = V1 - 32*DV), so only the schedule quantities that decide
// arithmetic -- the accumulated panel origins VFT_p, the far-wing window
// boundaries and which window each panel uses -- are planned on the host,
// in strict IEEE FP64 with the reference's operation order.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/lblgpu.h"

namespace lbl {

constexpr int kNMolTab = 7;     // HITRAN molecules with TIPS tables here
constexpr int kNIsoTab = 12;    // isotopologue slots (1-based, 11 used)
constexpr int kNfmx = 2601;     // NFMX, src/lblparams.f90:31
constexpr int kNShift = 32;     // NSHIFT
constexpr int kNlim1 = 2401;    // NLIM1
constexpr int kLimOut = 2500;   // LIMOUT of LBLF4
constexpr int kMaxSeg = 64;     // radiation segments per panel (RADFNI)

// Per-layer scalars the kernels read.  Plain data, copied to the device.
struct LayerDev {
  // /FILHDR/ and derived
  double pave, tave, dv, v1, v2, vft0;
  double xkt;                 // TAVE/RADCN2
  double betacr_n;            // LNCOR1: (1/XKT)-(1/XKT0)
  double beta_f, betacr_f;    // LINF4: RADCN2/TAVE, BETA-BETA0
  double tratio, rhorat, pavp0, pavp2;
  double rectlc_n, tmpdif_n, rectlc_f, tmpdif_f;
  int32_t ilc_n, ilc_f;       // line-coupling temperature brackets
  int32_t jrad, ilblf4, icntnm, nmol;
  // near wing (HIRAC1)
  double dptmn, dptfc, alfmax, bound, vbot, vtop;
  double dvr2, dvr3, conf2, conf3, wavdxf;
  int64_t max1;
  int64_t npts;               // output points
  int64_t npanel;
  // far wing (OPDPTH/LBLF4)
  double dvr4, bound4, v1l4, v2l4;
  int32_t nwin;
  int32_t pad0;
  // continuum grid (OPDPTH)
  double v1abs, v2abs, dvabs, h2o_fac;
  double wtot;                // WTOT of CONTNM: WBROAD + sum of WK
  int64_t nptabs;
  // molecular constants (MOLEC), 1-based molecule / isotopologue
  double wk[kNMolTab + 1];
  double scor[kNMolTab + 1][kNIsoTab];
  double rhoslf[kNMolTab + 1];
  double alfd1[kNMolTab + 1][kNIsoTab];
  int32_t isomax[kNMolTab + 1];
  // offsets of this layer's slices in the batch arrays
  int64_t off_r1, n_r1;       // R1 global index g1 in [1, n_r1]
  int64_t off_r2, n_r2;       // R2 g2 in [1, n_r2]
  int64_t off_r3, n_r3;       // R3 g3 in [1, n_r3]
  int64_t off_od;             // OD output (npts)
  int64_t off_panel;          // per-panel arrays (npanel entries)
  int64_t off_win;            // window table (nwin entries)
  int64_t off_r4;             // R4 storage (nwin * kR4Stride)
  int64_t off_far;            // raw far-wing line slots
  int64_t off_shr;            // shrunk line slots
  int64_t off_near;           // near-wing line slots
  int64_t off_nblk;           // near-range TAPE3 panel slots
  int64_t off_blk9;           // shrunk-line (TAPE9) block slots
  int64_t off_abs;            // continuum (ABSRB) slots
  int64_t off_seg;            // LINF4 segment slots (one per far-range panel)
  // line index ranges into the TAPE3 arrays
  int64_t far_lo, far_hi;     // [lo, hi) candidates for LINF4
  int64_t near_lo, near_hi;   // [lo, hi) candidates for RDLIN/LNCOR1
  int64_t blk_lo, blk_hi;     // TAPE3 panels spanned by the near range
  int64_t fblk_lo, fblk_hi;   // TAPE3 panels spanned by the far range
};

constexpr int64_t kR4Stride = kLimOut + 8;

// One LBLF4 call: window of NPTR4 points starting at V1R4.
struct WinDev {
  double v1r4, v2r4, vlo, vhi, vnulst, dptmn;
  int32_t nptr4;
  int32_t first_panel;        // first panel that uses this window
};

// Host-side plan of one layer.
struct LayerPlan {
  LayerDev d;
  std::vector<double> vft;      // VFT_p, p = 0..npanel-1
  std::vector<int32_t> win_of;  // window used by panel p
  std::vector<WinDev> win;
};

// Tables built once per context (host copies; uploaded by the library).
struct ShapeTables {
  double f1[kNfmx + 1], f2[kNfmx + 1], f3[kNfmx + 1], fg[kNfmx + 1], xver[kNfmx + 1];
};
void build_shape_tables(ShapeTables* t);

// PATH DV rule (src/lblrtm.f90:5355-5510).
int dv_rule(const lbl_run& R, lbl_layer* L, int nlay, std::string* err);
// Output points of a layer (PANEL last-panel rule).
int64_t layer_npts(const lbl_run& R, double dv);
// Host copy of the line fields the planner needs to find line ranges.
struct HostLines {
  const double* vnu;
  const float* sp;
  const float* pshift;
  const int32_t* mol;
  const int32_t* iflg;
  int64_t n;
  const int64_t* bs;   // TAPE3 panel starts, nblk+1 entries
  int64_t nblk;
  double max_abs_pshift;  // largest |PSHIFT| of the file
};
// Plan a layer; jrad is the sticky JRAD value entering OPDPTH.
int plan_layer(const lbl_run& R, const lbl_layer& L, int jrad,
               const HostLines& H, LayerPlan* P, std::string* err);
// JRAD after OPDPTH for this layer (src/lblrtm.f90:6211).
int next_jrad(const lbl_run& R, const lbl_layer& L, int jrad);

// PNLINT (src/oprop.f90:1564-1806) re-grids each 2400-point PANEL output to
// DVOUT as the panels stream past.  Which input panel computes an output
// point decides the point's interpolation coordinate (V1PO and V1P are both
// accumulated sums), so the host replays the reference's panel loop and
// hands the kernel one segment per (output panel, input panel) pair: output
// points ii_lo..ii_hi (1-based within the output panel that starts at
// global output index k0) are interpolated from input panel p, whose R1(1)
// is global layer point g0 = 2400*p.
struct PnlSeg {
  double v1po;                // V1PO of the output panel
  double v1p;                 // V1P of the input panel
  double fj1dif;              // FJ1DIF = (V1PO-V1P)/DVP+1+2
  int64_t k0;                 // global output index of the output panel's II=1
  int64_t g0;                 // global layer index of the input panel's R1(1)
  int32_t ii_lo, ii_hi;       // II range computed during this input panel
  int32_t nlim;               // NLIM of the input panel before the end pad
  int32_t flags;              // 1: first input panel, 2: last input panel
};
struct PnlPlan {
  std::vector<PnlSeg> seg;
  int64_t n_out = 0;          // output points of the layer
  bool copy = false;          // |DVOUT-DV| < 1e-8: panels pass through
  double a[4][101];           // Lagrange weights A1..A4 at P = 0.01*JP
};
// Plan PNLINT for a layer of spacing dv; dvout must satisfy 0 < dvout <= dv.
int pnlint_plan(const lbl_run& R, double dv, double dvout, PnlPlan* P, std::string* err);

// SCANFN (src/postsub.f90:25-560) on the global output grid: the scanning
// function table, SHRKSC's compression ratio and CONVSC's constants.
struct ScanPlan {
  int jfn = 0;
  double hwhm = 0., dvo = 0., hwf = 0., dxf = 0., bound = 0., vft0 = 0., vbot = 0., vtop = 0.;
  int64_t nf = 0, nfmax = 0, nnhi = 0;   // NNHI: last output point, R1 index
  int64_t n_out = 0;                     // output points (R1 33..NNHI)
  double bfov = 0.;                      // JFN 5/6: the field-of-view half angle, radians
  double dvint = 0.;                     // DVINT: coarser input is interpolated first
  std::vector<double> xf;                // XF, 1-based
  // compression and convolution for an input spacing
  int64_t iratsh = 1;
  double dvsc = 0., v1shft = 0., ratio = 0., zslope = 0., zbound = 0., xnorm = 0.;
};
// Grid, table and constants for input spacing dv_in.  A spacing above
// SCANFN's DVINT gives LBL_E_RANGE with P->dvint set: the spectrum is then
// first interpolated onto DVINT (scnint_plan) and planned again.
int scan_plan(const lbl_scan& sc, double dv_in, ScanPlan* P, std::string* err);

// SCNINT/INTERP (src/postsub.f90:824-1035, 2940-3215): the output points in
// chunks that carry the fraction P from point to point; each chunk starts
// from the wavenumber at its first point.  panel: the input panel (2400
// points) current in the chunk; i0, p0: INTERP's I (1-based in that
// panel's T array, T(5) its first point) and P at the chunk's first point;
// zero: points past the input, set to 0.
struct ScnChunk {
  int64_t out0, panel, i0;
  double p0;
  int32_t count, zero;
};
int scnint_plan(int64_t n, double v1_in, double dv_in, double dvo, std::vector<ScnChunk>* chunks,
                int64_t* n_fine, std::string* err);
// INTERP's weights C1..C4 at IP = 0..202 (P = (IP-1)/200), 4 x 203 values.
void scnint_coefs(double* c);

}  // namespace lbl
