/*
 * lblgpu.h -- C ABI of the B200 line-by-line layer optical-depth and
 * radiance-merge library.
 *
 * The entry points replace the per-layer calls that LBLRTM's layer loop
 * makes (src/lblrtm.f90 XLAYER, standard loop :3640-3657):
 *
 *   CALL OPDPTH (MPTS)                      -> lbl_layer_od
 *   CALL XMERGE (NPTS,LFILE,MFILE,JPATHL)   -> lbl_merge_layer
 *
 * plus whole-profile and many-profile forms of the same loop
 * (lbl_forward, lbl_forward_batch) and the radiance Jacobians
 * (lbl_jacobian), which the reference obtains from its IMRG=40-43
 * analytic-derivative workflow (src/lblrtm.f90:2855-3067).
 *
 * The reference passes everything through COMMON blocks (/FILHDR/,
 * /MANE/, /CNTSCL/) and disk files (TAPE3 lines, TAPE10 layer optical
 * depth, TAPE11/12 accumulated radiance).  Here the same quantities are
 * passed as plain structs and caller-owned buffers; every function returns
 * an lbl_status and never exits the process (the reference STOPs).
 *
 * Pointers marked "host or device" may point to either memory; the library
 * inspects them and copies as needed.  All functions are thread-safe on
 * distinct contexts; one context must not be used from two threads at once.
 */
#ifndef LBLGPU_H
#define LBLGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBL_WKDIM 60      /* /FILHDR/ WK(60), src/oprop.f90:107 */
#define LBL_MXMOL 47      /* MXMOL, src/lblparams.f90:28 */

typedef enum lbl_status {
  LBL_OK = 0,
  LBL_E_ARG = 1,          /* bad argument (NULL pointer, size, flag value) */
  LBL_E_UNSORTED = 2,     /* line centres not ascending (RDLIN assumes it) */
  LBL_E_NREC = 3,         /* a TAPE3 panel holds more than 250 lines
                             ('RDLIN; NREC GT LIMIN', src/oprop.f90:763) */
  LBL_E_ITYPE = 4,        /* layer DV ratio not allowed by the merge
                             (' RADMRG; ITYPE LT 0 ', src/xmerge.f90:2741) */
  LBL_E_CUDA = 5,         /* a CUDA runtime call failed */
  LBL_E_NOMEM = 6,        /* device or host allocation failed */
  LBL_E_RANGE = 7,        /* input outside the supported range (e.g. TIPS
                             temperature outside 70-3000 K, DV rule TYPE>2.5,
                             'PATH; ISTOP EQ 1' src/lblrtm.f90:5557) */
  LBL_E_NOTREADY = 8,     /* lines or tables not uploaded yet */
  LBL_E_CONVERGE = 9,     /* far-wing rejection fixpoint did not settle */
  LBL_E_FORMAT = 10,      /* malformed TAPE3 file */
  LBL_E_NODEVICE = 11     /* no CUDA device / library built without one */
} lbl_status;

/* Arithmetic of the line-shape, far-wing and merge kernels. */
typedef enum lbl_precision {
  LBL_PREC_FP64 = 0,      /* plain FP64 throughout: the drop-in form */
  LBL_PREC_SPLIT = 1      /* FP32 line shapes (near wing: FP32 values summed
                             per grid point with Kahan compensation; far
                             wing: FP32 per chunk of lines, added to an FP64
                             total) and FP32 merge; FP64 grid positions,
                             line-centre offsets, table indices and far-wing
                             rejection decisions */
} lbl_precision;

/* Run-level control: TAPE5 records 1.2, 1.2a, 1.3, 1.4 (subset on the hot
 * path).  Field names follow the reference variables. */
typedef struct lbl_run {
  int32_t ihirac;   /* 1: Voigt line shape (HIRAC1); the only value supported */
  int32_t ilblf4;   /* 0: no far wing; 1: F4 far wing with BOUND4=25 cm-1;
                       2: as 1 but BOUND4=5 cm-1 when PAVE<=0.5 mb
                       (src/lblrtm.f90:6246-6247) */
  int32_t icntnm;   /* 0: no continuum; 1: MT_CKD-style H2O self+foreign
                       (table from lbl_mtckd_upload) and Rayleigh
                       extinction (see xrayl) */
  int32_t iemit;    /* 0: optical depth only (ABINIT/ABSMRG);
                       1: radiance and transmittance (EMINIT/RADMRG) */
  int32_t ipathl;   /* 1: upwelling radiance, looking down (the first layer
                          the surface's, TMPBND/BNDEMI its emission);
                       2: the symmetric tangent path (IANT=0): the first
                          layer is the tangent layer, every layer is crossed
                          twice, its far crossing radiating at TZL (EMINIT
                          src/xmerge.f90:2442-2447, RADNN IPATH=2
                          :2997-3005, 3132-3148; TZL > 0 required);
                       3: downwelling radiance, looking up from the first
                          layer (RADNN IPATH=3, src/xmerge.f90:3007-3013,
                          3150-3166; TMPBND/BNDEMI a boundary beyond the
                          last layer, EMBND :3652-3733); Jacobians: 1 only */
  int32_t jrad;     /* initial JRAD: 1 (IRAD=0) or -1 (no radiation term),
                       src/lblrtm.f90:828-833 */
  double v1, v2;    /* spectral range, cm-1 (V2-V1 <= 2020 as in TAPE5 1.3) */
  double sample;    /* SAMPLE   (default 4)    */
  double dvset;     /* DVSET    (default 0)    */
  double alfal0;    /* ALFAL0   (default 0.04) */
  double avmass;    /* AVMASS   (default 36)   */
  double dptmin;    /* DPTMIN   (default 2e-4) */
  double dptfac;    /* DPTFAC   (default 1e-3) */
  double xself;     /* continuum scale factors, /CNTSCL/ (default 1) */
  double xfrgn;
  double tmpbnd;    /* boundary temperature TMPBND, K (record 1.4) */
  double bndemi;    /* boundary emissivity BNDEMI(1); BNDEMI(2:3)=0 */
  double xrayl;     /* Rayleigh scale XRAYL, /CNTSCL/ (default 1, 0 = off):
                       with ICNTNM=1 and V2 >= 820 cm-1 the continuum adds
                       Rayleigh extinction (src/contnm.f90:955-976) */
  double xco2c;     /* CO2 continuum scale XCO2C, /CNTSCL/ (default 1, 0 =
                       off): with ICNTNM=1 the continuum adds the CO2
                       continuum (src/contnm.f90:326-378, FRNCO2 :1295-1349)
                       between the H2O part and Rayleigh */
  double xo2cn;     /* O2 continuum scale XO2CN (default 1, 0 = off): the
                       collision-induced fundamental, 1340-1850 cm-1
                       (src/contnm.f90:491-540, o2_ver_1 :7254-7318), and
                       the 1.27 um band, 7536-8500 cm-1 (:543-584, O2INF1
                       :7384-7440) */
  double xn2cn;     /* N2 continuum scale XN2CN (default 1, 0 = off): the
                       collision-induced rotational band below 350 cm-1
                       (:745-792, xn2_r :2497-2566), fundamental,
                       2001.77-2897.59 cm-1 (:811-858, n2_ver_1 :2668-2754),
                       and first overtone, 4340-4910 cm-1 (:860-906,
                       n2_overtone1 :2916-2968) */
  double bndrfl;    /* boundary reflectivity BNDRFL(1) (record 1.4; default
                       0, BNDRFL(2:3)=0): with IPATHL=1 a value in (0, 1]
                       makes the run the reflected atmosphere (IBPROP=1,
                       IPATHL=-1, specular: EMINIT src/xmerge.f90:2486-2540,
                       RADNN IPATH=-10 :3023-3066, 3168-3215): each layer's
                       downward emission (at TZL) is reflected at the
                       surface and seen back up through the layers below */
} lbl_run;

/* One layer: the /FILHDR/ quantities OPDPTH and XMERGE read
 * (src/lblrtm.f90:4374-4412). */
typedef struct lbl_layer {
  double pave, tave;       /* layer pressure (mb) and temperature (K) */
  double pzl, pzu;         /* lower / upper level pressure (mb) */
  double tzl, tzu;         /* lower / upper level temperature (K) */
  double wk[LBL_WKDIM];    /* column amounts, molec/cm2; wk[m-1] is HITRAN
                              molecule m */
  double wbroad;           /* broadening-gas column, molec/cm2 */
  int32_t nmol;            /* molecules in use (<= LBL_MXMOL) */
  int32_t itype;           /* ITYL from the DV rule (output of lbl_dv_rule) */
  double dv;               /* layer DV, cm-1 (output of lbl_dv_rule) */
} lbl_layer;

/* TAPE3 line records in structure-of-arrays form, in file order
 * (struct_types.f90:106-125: VNU is REAL*8, the rest REAL*4/INTEGER*4).
 * Lines are grouped into TAPE3 panels of at most 250 records; the panel
 * boundaries matter to the far-wing line shrinking (LINF4) and to when
 * lines are read, so they are part of the input. */
typedef struct lbl_lines {
  int64_t n;
  const double*  vnu;      /* line centre, cm-1, ascending */
  const float*   sp;       /* strength, cm-1/(molec cm-2) at 296 K */
  const float*   alfa;     /* air-broadened HWHM at 296 K, 1013 mb */
  const float*   epp;      /* lower-state energy, cm-1 */
  const int32_t* mol;      /* ISO*100 + MOL */
  const float*   hwhms;    /* self-broadened HWHM */
  const float*   tmpalf;   /* temperature exponent of the width */
  const float*   pshift;   /* pressure shift, cm-1/atm */
  const int32_t* iflg;     /* line flag; <0 records are coupling data */
  int64_t nblock;          /* number of TAPE3 panels, 0 = consecutive 250 */
  const int64_t* block_start; /* nblock+1 offsets into the arrays, or NULL */
} lbl_lines;

/* MT_CKD-style H2O continuum coefficient table on a uniform grid, the
 * layout of absco-ref_wv-mt-ckd.nc read by mt_ckd_h2o_module.f90:68-174. */
typedef struct lbl_mtckd {
  int64_t n;
  double v0, dv;                 /* wavenumber of entry 0 and spacing */
  const double* self_absco_ref;  /* cm2/molec/cm-1 at ref_press/ref_temp */
  const double* for_absco_ref;
  const double* self_texp;
  double ref_press, ref_temp;    /* 1013 mb, 296 K in the reference file */
} lbl_mtckd;

typedef struct lbl_ctx lbl_ctx;

/* ---- context ---------------------------------------------------------- */

/* Create a context on CUDA device `device`; builds the line-shape tables
 * (SHAPEL/SHAPEG/VERFN, src/oprop.f90:1822-1991) on the device. */
int lbl_ctx_create(int device, lbl_ctx** out);
int lbl_ctx_destroy(lbl_ctx* ctx);
/* Last error message of this context (empty if none). */
const char* lbl_last_error(const lbl_ctx* ctx);
/* Set the CUDA stream (cudaStream_t) used by later calls; NULL = default.
 * The context also owns two internal non-blocking streams (created on first
 * use): on one, the kernels that need only the layer plans run beside the
 * far wing, and results are copied out while the last merge launch runs
 * (joined to the caller's stream by events); on the other, each group of
 * lbl_forward_batch is captured as a CUDA graph, which is then launched on
 * the caller's stream.  Every call that returns results synchronises before
 * it returns. */
int lbl_set_stream(lbl_ctx* ctx, void* stream);

/* Cap the device memory the context holds (lines, tables, work arenas,
 * merge and Jacobian buffers) at `bytes`; 0 removes the cap.  The context's
 * grow-only work buffers are released (after its stream is idle) and
 * allocated again within the cap by later calls.  A call that would need
 * more returns LBL_E_NOMEM (as when the device itself is full) and leaves
 * the context usable.  The batched calls size their groups of profiles, and
 * the Jacobians their chunks of parameters, to fit under the cap. */
int lbl_set_memory_limit(lbl_ctx* ctx, int64_t bytes);
/* Device memory the context holds now, in bytes (-1 for a NULL context). */
int64_t lbl_memory_used(const lbl_ctx* ctx);

/* ---- inputs ----------------------------------------------------------- */

/* Copy the TAPE3 line records (host arrays) to the device, where they stay
 * resident.  Replaces opening TAPE3 on unit LINFIL (src/lblrtm.f90:801-808)
 * and the per-layer re-reads of RDLIN (src/oprop.f90:678).  Fails with
 * LBL_E_UNSORTED / LBL_E_NREC on the conditions RDLIN assumes or STOPs on. */
int lbl_lines_upload(lbl_ctx* ctx, const lbl_lines* lines);

/* Read a TAPE3 file (Fortran unformatted, 4-byte record markers, the
 * INPUT_HEADER/INPUT_BLOCK records of struct_types.f90:106-125) and upload
 * it.  Returns the number of line records through *nlines (may be NULL).
 * A truncated or malformed record gives LBL_E_FORMAT, a panel of more than
 * 250 records LBL_E_NREC, descending centres LBL_E_UNSORTED.  With ctx NULL
 * the file is read and checked the same way but nothing is uploaded (no
 * device is needed). */
int lbl_lines_load_tape3(lbl_ctx* ctx, const char* path, int64_t* nlines);

/* Upload the H2O continuum coefficient table (CONTNM, contnm.f90:279-324). */
int lbl_mtckd_upload(lbl_ctx* ctx, const lbl_mtckd* table);

/* ---- host-side planning (no device work) ------------------------------ */

/* The per-layer DV rule of PATH (src/lblrtm.f90:5407-5510): fills
 * layers[l].dv and layers[l].itype for l = 0..nlay-1 in path order. */
int lbl_dv_rule(const lbl_run* run, lbl_layer* layers, int32_t nlay);

/* Number of points OPDPTH writes for a layer of spacing dv: the panels of
 * PANEL (src/oprop.f90:1435-1451) end at the first grid point >= V2. */
int64_t lbl_layer_npts(const lbl_run* run, double dv);

/* ---- one layer: OPDPTH ------------------------------------------------ */

/* Monochromatic optical depth of one layer on its own grid
 * v_i = V1 + i*dv, i = 0..npts-1 (TAPE10 content, src/lblrtm.f90:6135).
 * *jrad is the sticky JRAD flag (FSCDID(9)); it is read and updated as
 * OPDPTH does (src/lblrtm.f90:6211).  od: host or device, npts doubles. */
int lbl_layer_od(lbl_ctx* ctx, const lbl_run* run, const lbl_layer* layer,
                 int32_t* jrad, double* od, int64_t npts, int32_t precision);

/* ---- optical depth on a DVOUT grid: PNLINT ---------------------------- */

/* Points PNLINT writes (src/oprop.f90:1564-1806, called from PANEL
 * :1524-1532 when /IODFLG/ DVOUT is nonzero) for a layer of spacing dv
 * re-gridded to dvout: output panels of up to 2400 points from V1 in steps
 * of dvout, ending at the first point >= V2.  |dvout-dv| < 1e-8 passes the
 * layer grid through (lbl_layer_npts points).  Negative: minus a status
 * (-LBL_E_ARG, also for dvout > dv: the reference prints "DVOUT MUST BE <
 * DV", src/lblrtm.f90:5567-5568, and then reads past its panel buffer). */
int64_t lbl_pnlint_npts(const lbl_run* run, double dv, double dvout);

/* PNLINT: the layer optical depth od_in (n_in = lbl_layer_npts(run, dv)
 * points on V1 + i*dv, as lbl_layer_od writes it) interpolated to the DVOUT
 * grid with the reference's 4-point Lagrange weights tabulated at 1/100 of
 * dv (n_out = lbl_pnlint_npts points).  Reproduces the reference's
 * streaming order: each output point takes its interpolation coordinate
 * from the PANEL panel that was current when the reference computed it.
 * This is the layer output of IOD=1/4 (DVOUT from DVSET) and of the IOD=3
 * common grid.  od_in, od_out: host or device. */
int lbl_pnlint(lbl_ctx* ctx, const lbl_run* run, double dv, double dvout,
               const double* od_in, int64_t n_in, double* od_out, int64_t n_out);

/* ---- instrument scanning function: SCANFN ---------------------------- */

/* SCANFN's scanning functions (src/postsub.f90:25-560, CONVSC :1516-1598,
 * SHRKSC :1276-1376, shapes SHAPET :1377, SHAPEG src/oprop.f90:1912,
 * SINCSQ :2445, SINC :2486; the rectangle CNVRCT :1779-1985, the
 * field-of-view boxes CNVVRC :1986-2214 and CNVVRL :2216-2440) convolved
 * with a spectrum on a uniform grid. */
typedef struct lbl_scan {
  double hwhm;      /* HWHM of the function, cm-1 (JFN -3/-4: its first
                       zero crossing, divided by pi/XSCALE as SCANFN does;
                       JFN 5/6: the field of view's half angle, degrees) */
  double v1, v2;    /* output range, cm-1 */
  double sampl;     /* SAMPL: > 0 points per HWHM, < 0 minus the output
                       spacing, 0 the function's default (2 or 4) */
  int32_t jfn;      /* 0 rectangle, 1 triangle, 2 Gaussian, 3 sinc^2,
                       4 sinc, 5 boxes of width V*B^2/2 centred at the
                       output points, 6 the same boxes starting there
                       (B the half angle in radians); -3, -4 */
  int32_t jabs;     /* 1: convolve 1 - spectrum (JEMIT=-1, absorption) */
} lbl_scan;

/* Output points and spacing of lbl_scan_spectrum for an input spacing
 * dv_in: points V1 + j*DVOUT up to the one nearest V2 (PANLSC's last panel,
 * :1600-1660); for the rectangle, DVOUT = IRATIO*dv_in with IRATIO the
 * nearest whole number to HWHM/(SAMPLE*dv_in), and the boxes centred at
 * V1 + j*DVOUT <= V2.  An input spacing above SCANFN's DVINT (HWHM/12; for
 * JFN 5/6 V1*B^2/24) is first interpolated onto DVINT as the reference does
 * (SCNINT/INTERP, src/postsub.f90:824-1035, 2940-3215), and the grid is that
 * of DVINT.  Negative: minus a status (-LBL_E_ARG for a bad argument,
 * -LBL_E_RANGE when the rectangle's IRATIO is below 2). */
int64_t lbl_scan_npts(const lbl_scan* sc, double dv_in, double* dvout);

/* The scanned spectrum: spec on v1_in + i*dv_in (n points, host or device),
 * compressed by SHRKSC's integer ratio, convolved as CONVSC does (each
 * output point the sum, in input order, of XNORM*S(I)*XF(IT) over the
 * inputs whose function reaches it), on the global output grid (the
 * reference's panel origins and incremental table offsets round slightly
 * differently; see lbl_scan_npts for the grid).  The rectangle (JFN 0)
 * (and JFN 5/6) is CNVRCT's weighted box mean: the inner points weight 1,
 * the two end points the fraction of their interval inside the box; every
 * box must
 * lie inside the input (LBL_E_RANGE otherwise).  out: n_out points, host
 * or device. */
int lbl_scan_spectrum(lbl_ctx* ctx, const lbl_scan* sc, const double* spec, int64_t n,
                      double v1_in, double dv_in, double* out, int64_t n_out);

/* ---- one merge step: XMERGE ------------------------------------------ */

/* Merge one layer's optical depth into the accumulated radiance and
 * transmittance (XMERGE IEMIT=1: EMINIT for the first layer, RADMRG/RADNN
 * after, src/xmerge.f90:25-167; IEMIT=0: ABINIT/ABSMRG).
 *   first         bit 0: the first layer (EMINIT); bit 1: the last layer,
 *                 which looking up (IPATHL=3) adds the boundary beyond it
 *                 (XMERGE :136-141)
 *   od            layer optical depth, n_new points (host or device)
 *   rad_in/tr_in  accumulated radiance/transmittance on the previous
 *                 layer's grid, n_old points (ignored for the first layer)
 *   rad_out/tr_out results on the layer grid, n_new points
 * For IEMIT=0 rad_* carry accumulated optical depth and tr_* is unused. */
int lbl_merge_layer(lbl_ctx* ctx, const lbl_run* run, const lbl_layer* layer,
                    int32_t first, double dv_old, const double* rad_in,
                    const double* tr_in, int64_t n_old, const double* od,
                    double* rad_out, double* tr_out, int64_t n_new);

/* ---- one merge step without any allocation ------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory -- where a caching allocator owns the device, or the call sits in
 * a region that must not grow the memory footprint, or a host framework
 * only hands out buffers it already owns.  Runs the same merge kernel as
 * lbl_merge_layer on device `device` and CUDA stream `stream` (NULL =
 * default), with no context: od, rad_in, tr_in, rad_out and tr_out must all
 * be caller-owned memory of device `device` (host pointers or another
 * GPU's memory give LBL_E_ARG), and the call allocates nothing.  An output
 * must not share memory with rad_in, tr_in or the other output (LBL_E_ARG);
 * it may be od itself.  IEMIT must be 0 or 1, IPATHL 1 (no reflectivity) and first 0 or 1;
 * with IEMIT=0 tr_in and tr_out are not used.  Its only scratch is a
 * fixed device array inside the library, about 72 KB on every device that
 * loads it, kept until the
 * process exits; it bounds a layer to LBL_NOALLOC_MAX_PANELS panels of 2400
 * points (19,660,800 points); longer layers return LBL_E_RANGE.  The first
 * call on a device looks up that array's device address; make that first
 * call before any stream capture on the device.  Every call rewrites all of
 * the scratch it reads, but all calls share the one array: calls that
 * overlap on the GPU (different host threads or streams) race.  The caller's
 * current device is restored before the call returns, and the call returns
 * after its stream has finished the merge. */
#define LBL_NOALLOC_MAX_PANELS 8192
int lbl_merge_layer_noalloc(int device, const lbl_run* run, const lbl_layer* layer,
                            int32_t first, double dv_old, const double* rad_in,
                            const double* tr_in, int64_t n_old, const double* od,
                            double* rad_out, double* tr_out, int64_t n_new, void* stream);

/* ---- whole path ------------------------------------------------------- */

/* The standard layer loop (XLAYER :3640-3657) for one profile: DV rule,
 * OPDPTH per layer, XMERGE per layer.  Outputs on the last layer's grid
 * (lbl_layer_npts of layers[nlay-1].dv points, host or device):
 *   rad: upwelling radiance at the top (W/(cm2 sr cm-1)), IEMIT=1, or total
 *        optical depth, IEMIT=0;  tr: total transmittance (may be NULL).
 * layers[].dv/itype are computed here (lbl_dv_rule) and written back. */
int lbl_forward(lbl_ctx* ctx, const lbl_run* run, lbl_layer* layers,
                int32_t nlay, double* rad, double* tr, int64_t npts,
                int32_t precision);

/* Many independent profiles (uneven layer counts) in one call.  layers is
 * the concatenation of all profiles' layers; nlay[p] is profile p's count.
 * rad/tr are concatenated per profile; offsets[p] (output, nprof+1 entries)
 * gives where profile p starts; npts_total bounds the buffers. */
int lbl_forward_batch(lbl_ctx* ctx, const lbl_run* run, lbl_layer* layers,
                      const int32_t* nlay, int32_t nprof, double* rad,
                      double* tr, int64_t* offsets, int64_t npts_total,
                      int32_t precision);

/* Jacobians of the top-of-atmosphere radiance of one profile with respect
 * to each layer's temperature (K) and the log column amount of the listed
 * molecules (the reference's analytic-Jacobian path, IMRG=40-43: layer
 * optical-depth derivatives TDERIVup/QDERIVup, merge derivatives EMDT/
 * EMADMG, src/xmerge.f90:4406-6144).  Optical-depth derivatives are central
 * differences (T +-0.1 K, amount +-1 %) of two whole-profile passes per
 * parameter; the merge is differentiated by hand and each layer's row is
 * carried to the top through the later layers' transmittance and grid
 * changes.  Upwelling radiance only (IEMIT=1, IPATHL=1); at most 7 molecules.
 * Output layout (host or device):
 *   jac[(k*nlay + l)*npts + i]  k=0: d rad_i / d T_l,
 *                               k=1..nq: d rad_i / d ln W_{mols[k-1]},l
 * on the last layer's grid.  rad (optional) receives the forward result.
 * layers[].dv/itype are computed here (lbl_dv_rule) and written back. */
int lbl_jacobian(lbl_ctx* ctx, const lbl_run* run, lbl_layer* layers,
                 int32_t nlay, const int32_t* mols, int32_t nq, double* rad,
                 double* jac, int64_t npts, int32_t precision);

/* How the batched Jacobians obtain a layer's optical-depth derivatives. */
typedef enum lbl_jac_mode {
  LBL_JAC_CENTRAL = 0,    /* central differences (T +-0.1 K, amount +-1 %)
                             merged with the exact derivative of the merge:
                             the derivative of the discrete forward model */
  LBL_JAC_REFERENCE = 1   /* the reference's analytic-Jacobian definitions
                             (src/lblrtm.f90:2855-3067): a pass at T + 1 K and
                             one per molecule with that molecule alone (other
                             amounts zero, WK(7) added to WBROAD), merged by
                             the TDERIVup/QDERIVup rows (src/xmerge.f90:
                             5786-6144) from the quantities EMDT saves */
} lbl_jac_mode;

/* Forward and Jacobians of many profiles (uneven layer counts) in one call:
 * the batched form of the reference's analytic-Jacobian run.  Each profile
 * costs one optical-depth pass per derivative pass (LBL_JAC_REFERENCE:
 * 1 + nq after the nominal one; LBL_JAC_CENTRAL: 2 (1 + nq)) queued back to
 * back without host waits, then one merge sweep that forms every layer's
 * row and carries it to the top through the later layers.  When a
 * profile's work space for all parameters would not fit the device (or the
 * lbl_set_memory_limit cap), the parameters are taken in chunks and the
 * nominal pass is recomputed for each chunk.
 *   dv_chan > 0: radiance and Jacobians are averaged over channels
 *     [V1 + c dv_chan, V1 + (c+1) dv_chan), c < floor((V2-V1)/dv_chan) (a
 *     boxcar instrument function); dv_chan = 0: each profile's top grid.
 *   rad: concatenated per profile, profile p at offsets[p] (nprof+1
 *        entries, output), rad_cap doubles available;
 *   jac: profile p's block jac[jac_off[p] + (k*nlay[p] + l)*n_p + i]
 *        (k = 0: d/dT_l, k = 1..nq: d/d ln W_{mols[k-1],l}), jac_off output
 *        (nprof+1 entries), jac_cap doubles available.
 * Host or device buffers; upwelling radiance only. */
int lbl_adjoint_batch(lbl_ctx* ctx, const lbl_run* run, lbl_layer* layers,
                      const int32_t* nlay, int32_t nprof, const int32_t* mols,
                      int32_t nq, int32_t mode, double dv_chan, double* rad,
                      int64_t* offsets, int64_t rad_cap, double* jac,
                      int64_t* jac_off, int64_t jac_cap, int32_t precision);

/* ---- timing and work counters ------------------------------------------
 * Per-stage device time, launch count and algorithmic work of the calls
 * made since the last read -- the counterpart of the per-layer timing table
 * HIRAC1 prints to TAPE6 (READ / CONVOLUTION / PANEL, src/oprop.f90:552-631).
 * Stage times are taken with CUDA events on the context's stream only while
 * profiling is enabled; launch counts and work are always recorded.
 * work units: far_wing = line-point evaluations of F4 (CONVF4 loop 40/45);
 * grids = near-wing point triples (CNVFNV loop 10); combine/merge = layer
 * points. */
typedef struct lbl_stage_stat {
  char name[24];
  double ms;           /* summed device time, 0 when profiling is off */
  int64_t launches;    /* kernel launches */
  double work;         /* algorithmic work units (see above) */
} lbl_stage_stat;

int lbl_profile(lbl_ctx* ctx, int32_t enable);
/* Copy up to cap stage records into out, set *n, and reset the counters. */
int lbl_profile_read(lbl_ctx* ctx, lbl_stage_stat* out, int32_t cap, int32_t* n);

/* Brightness temperature of a radiance spectrum (TEM, src/pltlbl.f90:1568):
 * bt_i = RADCN2*v_i / ln(RADCN1*v_i^3/rad_i + 1).  Host arrays. */
int lbl_brightness_temperature(const double* rad, int64_t n, double v1,
                               double dv, double* bt);

#ifdef __cplusplus
}
#endif
#endif /* LBLGPU_H */
