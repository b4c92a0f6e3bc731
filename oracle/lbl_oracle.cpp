// lbl_oracle.cpp -- CPU FP64 restatement of LBLRTM's layer optical-depth and
// radiance-merge path, used ONLY as test infrastructure (the checker for the
// CUDA library, and the timed CPU baseline of bench.py).  Nothing in the
// product links or calls this file.
//
// Parity status: the Fortran reference cannot be built here (no Fortran
// compiler; its aer_rt_utils I/O submodule and netCDF-Fortran are absent), so
// this restatement is pinned only by known-answer tests derived from the
// reference's own arithmetic (line-shape normalisation, partition-sum
// identities, DV-rule values, radiative-transfer limits) -- parity is
// partially pinned, not pinned against reference outputs.
//
// The restatement follows the reference routine by routine and keeps its
// sequential panel structure, Fortran integer truncation and FP64 ("dbl"
// build, build/makefile.common:217-221) arithmetic, so that a reader can
// check it against the Fortran line by line.  File I/O is replaced by
// in-memory "files": TAPE3 panels (lbl_lines + panel offsets), TAPE9 shrunk
// line blocks, TAPE10 layer panels and the merge panels.
//
// Routines restated (all paths relative to the LBLRTM source tree):
//   PATH DV rule        src/lblrtm.f90:5355-5510
//   OPDPTH              src/lblrtm.f90:6135-6287
//   HIRAC1              src/oprop.f90:25-633
//   RDLIN               src/oprop.f90:678-885
//   LNCOR1              src/oprop.f90:886-1197
//   CNVFNV              src/oprop.f90:1200-1370
//   PANEL               src/oprop.f90:1371-1561
//   SHAPEL/SHAPEG/VERFN src/oprop.f90:1822-1991
//   RSYM, XINT          src/oprop.f90:2145-2234
//   RADFN, RADFNI       src/oprop.f90:2235-2475
//   MOLEC               src/oprop.f90:2476-2557
//   LINF4, RDLNFL       src/oprop.f90:2934-3507
//   SHRINK              src/oprop.f90:3508-3640
//   LBLF4, RDLIN4       src/oprop.f90:3641-3832
//   CONVF4              src/oprop.f90:3833-4039
//   TIPS_2003, AtoB     src/oprop.f90:5919-6294, 11708-11798
//   CONTNM (H2O)        src/contnm.f90:199-324
//   mt_ckd_h2o_absco    src/mt_ckd_h2o_module.f90:68-296
//   XMERGE dispatch     src/xmerge.f90:25-167
//   ABINIT/ABSMRG       src/xmerge.f90:270-682
//   PLANCK              src/xmerge.f90:968-1017
//   EMIN                src/xmerge.f90:1684-1880 (LTE, IAERSL=0 branch)
//   EMINIT              src/xmerge.f90:2245-2583 (IPATHL=1, TBND>0 branch)
//   RADMRG/RADNN        src/xmerge.f90:2587-3130 (IPATH=1 branches)
//   TEM (BT)            src/pltlbl.f90:1567-1568

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <functional>
#include <vector>

#include "../include/lblgpu.h"
#include "../lblrtm_b200/data/ref_tables.h"
#include "../lblrtm_b200/data/cont_tables.h"

namespace {

// ---- constants (src/phys_consts.f90:66-74, src/lblrtm.f90:631-634) -------
const double PI = 3.1415926535898;
const double BOLTZ = 1.3806503E-16;
const double CLIGHT = 2.99792458E+10;
const double AVOGAD = 6.02214199E+23;
const double RADCN1 = 1.191042722E-12;
const double RADCN2 = 1.4387752;
const double ONEPL = 1.001, ONEMI = 0.999;
const double P0 = 1013.25, TEMP0 = 296.;  // src/lblrtm.f90:2115-2116
const double OD_LO = 0.06;                 // src/lblparams.f90:47

// Fortran INT() of a real: truncation toward zero.
inline long fint(double x) { return (long)x; }

std::string g_err;
// RSYM is always applied as the reference does; a test switches it off to
// show that the fold changes the lowest points of a run starting near zero.
bool g_rsym = true;
int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

// ---- line-shape sub-functions (SHAPEL, SHAPEG, VERFN) --------------------
// 1-based arrays of NFMX = 2601 entries (src/lblparams.f90:31).
const int NFPTS = 2001, NFMX = 2601;
const double HWF1 = 4., DXF1 = 0.002, HWF2 = 16., DXF2 = 0.008, HWF3 = 64.,
             DXF3 = 0.032;
const int NX1 = NFPTS, NX2 = NFPTS, NX3 = NFPTS;

struct Shapes {
  double F1[NFMX + 1], F2[NFMX + 1], F3[NFMX + 1], FG[NFMX + 1],
      XVER[NFMX + 1];
  Shapes() {
    // SHAPEL, src/oprop.f90:1822-1911
    auto A = [](double z0) { return (1. + 2. * z0 * z0) / std::pow(1. + z0 * z0, 2); };
    auto B = [](double z0) { return -1. / std::pow(1. + z0 * z0, 2); };
    double RECPI = 1. / (2. * std::asin(1.));
    double A1 = A(HWF1), B1 = B(HWF1), A2 = A(HWF2), B2 = B(HWF2), A3 = A(HWF3),
           B3 = B(HWF3);
    auto XL = [](double x) { return 1. / (1. + x); };
    auto Q1 = [&](double x) { return A1 + B1 * x; };
    auto Q2 = [&](double x) { return A2 + B2 * x; };
    auto Q3 = [&](double x) { return A3 + B3 * x; };
    for (int i = 0; i <= NFMX; i++) F1[i] = F2[i] = F3[i] = FG[i] = XVER[i] = 0.;
    F1[1] = RECPI * (XL(0.) - Q1(0.));
    for (int jj = 2; jj <= NX1; jj++) {
      double x = double(jj - 1) * DXF1, xsq = x * x;
      F1[jj] = RECPI * (XL(xsq) - Q1(xsq));
    }
    F1[NX1] = 0.;
    F2[1] = RECPI * (Q1(0.) - Q2(0.));
    long j1lim = fint(HWF1 / DXF2 + 1.001);
    for (long jj = 2; jj <= j1lim; jj++) {
      double x = double(jj - 1) * DXF2, xsq = x * x;
      F2[jj] = RECPI * (Q1(xsq) - Q2(xsq));
    }
    for (long jj = j1lim + 1; jj <= NX2; jj++) {
      double x = double(jj - 1) * DXF2, xsq = x * x;
      F2[jj] = RECPI * (XL(xsq) - Q2(xsq));
    }
    F2[NX2] = 0.;
    F3[1] = RECPI * (Q2(0.) - Q3(0.));
    long j2lim = fint(HWF2 / DXF3 + 1.001);
    for (long jj = 2; jj <= j2lim; jj++) {
      double x = double(jj - 1) * DXF3, xsq = x * x;
      F3[jj] = RECPI * (Q2(xsq) - Q3(xsq));
    }
    for (long jj = j2lim + 1; jj <= NX3; jj++) {
      double x = double(jj - 1) * DXF3, xsq = x * x;
      F3[jj] = RECPI * (XL(xsq) - Q3(xsq));
    }
    // SHAPEG, src/oprop.f90:1912-1942
    double FLN2 = std::log(2.);
    double FGNORM = std::sqrt(FLN2 * RECPI);
    FG[1] = FGNORM * std::exp(-FLN2 * 0.);
    for (int jj = 2; jj <= NX1; jj++) {
      double x = double(jj - 1) * DXF1, xsq = x * x;
      FG[jj] = FGNORM * std::exp(-FLN2 * xsq);
    }
    FG[NX1] = 0.;
    // VERFN, src/oprop.f90:1943-1991 (evaluated over all N1MAX entries)
    const double CEXP = 0.45, CE0 = 1., CE2 = -.20737285249, CE4 = -.00872684335747;
    double SE0 = std::sqrt(CEXP / PI);
    double AE2 = 2. * CEXP;
    double AE4 = AE2 * AE2 / 3.;
    for (int i = 1; i <= NFMX; i++) {
      double z = DXF1 * double(i - 1), z2 = z * z;
      double xe0 = SE0 * std::exp(-CEXP * z2);
      XVER[i] = (1. / (CE0 + CE2 + CE4)) * (CE0 + CE2 * AE2 * z2 + CE4 * AE4 * z2 * z2) * xe0;
    }
  }
};
const Shapes& shapes() {
  static Shapes s;
  return s;
}

// VOICON tables, 1-based (src/oprop.f90:1993-2144)
inline double AVRAT(long i) { return LBL_AVRAT[i - 1]; }
inline double CGAUSS(long i) { return LBL_CGAUSS[i - 1]; }
inline double CF1(long i) { return LBL_CF1[i - 1]; }
inline double CF2(long i) { return LBL_CF2[i - 1]; }
inline double CF3(long i) { return LBL_CF3[i - 1]; }
inline double CER(long i) { return LBL_CER[i - 1]; }

// ---- RADFN, RADFNI (src/oprop.f90:2235-2475) ----------------------------
double RADFN(double VI, double XKT) {
  double XVI = VI;
  if (XKT > 0.0) {
    double XVIOKT = XVI / XKT;
    if (XVIOKT <= 0.01) return 0.5 * XVIOKT * XVI;
    if (XVIOKT <= 10.0) {
      double EXPVKT = std::exp(-XVIOKT);
      return XVI * (1. - EXPVKT) / (1. + EXPVKT);
    }
    return XVI;
  }
  return XVI;
}

double RADFNI(double VI, double DVI, double XKT, double& VINEW, double& RDEL,
              double& RDLAST) {
  const double FACT1 = 3.0E-03;
  double XVI = VI;
  if (RDLAST < 0.) RDLAST = RADFN(XVI, XKT);
  double result = RDLAST;
  long INTVLS = 1;
  double RDNEXT;
  if (XKT > 0.0) {
    double XVIOKT = XVI / XKT;
    if (XVIOKT <= 0.01) {
      if (VINEW >= 0.0) {
        VINEW = VI + FACT1 * 0.5 * XVI;
        INTVLS = fint((VINEW - VI) / DVI);
        INTVLS = std::max(INTVLS, 1L);
        VINEW = VI + DVI * double(INTVLS);
      } else {
        VINEW = std::fabs(VINEW);
        INTVLS = fint((VINEW - VI) / DVI);
        INTVLS = std::max(INTVLS, 1L);
      }
      double XVINEW = VINEW;
      double XVINEWOKT = XVINEW / XKT;
      RDNEXT = 0.5 * XVINEWOKT * XVINEW;
    } else if (XVIOKT <= 10.0) {
      double EXPVKT = std::exp(-XVIOKT);
      double XMINUS = 1. - EXPVKT;
      double XPLUS = 1. + EXPVKT;
      if (VINEW >= 0.0) {
        double CVIKT = XVIOKT * EXPVKT;
        VINEW = VI + FACT1 * XVI / (1. + (CVIKT / XMINUS + CVIKT / XPLUS));
        INTVLS = fint((VINEW - VI) / DVI);
        INTVLS = std::max(INTVLS, 1L);
        VINEW = VI + DVI * double(INTVLS);
      } else {
        VINEW = std::fabs(VINEW);
        INTVLS = fint((VINEW - VI) / DVI);
        INTVLS = std::max(INTVLS, 1L);
      }
      double XVINEW = VINEW;
      double XVINEWOKT = XVINEW / XKT;
      double EXPVNEWKT = std::exp(-XVINEWOKT);
      RDNEXT = XVINEW * (1. - EXPVNEWKT) / (1. + EXPVNEWKT);
    } else {
      if (VINEW >= 0.0) {
        VINEW = VI + (FACT1 * XVI);
        INTVLS = fint((VINEW - VI) / DVI);
        INTVLS = std::max(INTVLS, 1L);
        VINEW = VI + DVI * double(INTVLS);
      } else {
        VINEW = std::fabs(VINEW);
        INTVLS = fint((VINEW - VI) / DVI);
        INTVLS = std::max(INTVLS, 1L);
      }
      RDNEXT = VINEW;
    }
  } else {
    if (VINEW >= 0.0) {
      VINEW = VI + (FACT1 * XVI);
      INTVLS = fint((VINEW - VI) / DVI);
      INTVLS = std::max(INTVLS, 1L);
      VINEW = VI + DVI * double(INTVLS);
    } else {
      VINEW = std::fabs(VINEW);
      INTVLS = fint((VINEW - VI) / DVI);
      INTVLS = std::max(INTVLS, 1L);
    }
    RDNEXT = VINEW;
  }
  RDEL = (RDNEXT - result) / double(INTVLS);
  RDLAST = RDNEXT;
  return result;
}

// ---- TIPS_2003 / AtoB (src/oprop.f90:5919-6294, 11708-11798) ------------
double AtoB(double aa, const double* A, const double* B, int npt) {
  // 1-based view
  auto a = [&](int i) { return A[i - 1]; };
  auto b = [&](int i) { return B[i - 1]; };
  auto nz = [](double d) { return d == 0. ? 0.0001 : d; };
  for (int I = 2; I <= npt; I++) {
    if (a(I) >= aa) {
      if (I < 3 || I == npt) {
        int J = I;
        if (I < 3) J = 3;
        if (I == npt) J = npt;
        double A0D1 = nz(a(J - 2) - a(J - 1)), A0D2 = nz(a(J - 2) - a(J));
        double A1D1 = nz(a(J - 1) - a(J - 2)), A1D2 = nz(a(J - 1) - a(J));
        double A2D1 = nz(a(J) - a(J - 2)), A2D2 = nz(a(J) - a(J - 1));
        double A0 = (aa - a(J - 1)) * (aa - a(J)) / (A0D1 * A0D2);
        double A1 = (aa - a(J - 2)) * (aa - a(J)) / (A1D1 * A1D2);
        double A2 = (aa - a(J - 2)) * (aa - a(J - 1)) / (A2D1 * A2D2);
        return A0 * b(J - 2) + A1 * b(J - 1) + A2 * b(J);
      }
      int J = I;
      double A0D1 = nz(a(J - 2) - a(J - 1)), A0D2 = nz(a(J - 2) - a(J)),
             A0D3 = nz(a(J - 2) - a(J + 1));
      double A1D1 = nz(a(J - 1) - a(J - 2)), A1D2 = nz(a(J - 1) - a(J)),
             A1D3 = nz(a(J - 1) - a(J + 1));
      double A2D1 = nz(a(J) - a(J - 2)), A2D2 = nz(a(J) - a(J - 1)),
             A2D3 = nz(a(J) - a(J + 1));
      double A3D1 = nz(a(J + 1) - a(J - 2)), A3D2 = nz(a(J + 1) - a(J - 1)),
             A3D3 = nz(a(J + 1) - a(J));
      double A0 = (aa - a(J - 1)) * (aa - a(J)) * (aa - a(J + 1));
      A0 = A0 / (A0D1 * A0D2 * A0D3);
      double A1 = (aa - a(J - 2)) * (aa - a(J)) * (aa - a(J + 1));
      A1 = A1 / (A1D1 * A1D2 * A1D3);
      double A2 = (aa - a(J - 2)) * (aa - a(J - 1)) * (aa - a(J + 1));
      A2 = A2 / (A2D1 * A2D2 * A2D3);
      double A3 = (aa - a(J - 2)) * (aa - a(J - 1)) * (aa - a(J));
      A3 = A3 / (A3D1 * A3D2 * A3D3);
      return A0 * b(J - 2) + A1 * b(J - 1) + A2 * b(J) + A3 * b(J + 1);
    }
  }
  return 0.;  // aa above the table: the Fortran leaves bb undefined
}

// Q(T) for (mol, iso); molecules outside 1..7 are not tabulated here.
bool tips_q(int mol, int iso, double T, double* q) {
  if (mol < 1 || mol > LBL_NQMOL || iso < 1 || iso > LBL_QNISO[mol - 1]) return false;
  if (T < 70. || T > 3000.) return false;
  *q = AtoB(T, LBL_TDAT, LBL_QOFT[mol - 1][iso - 1], 119);
  return true;
}

// ---- per-layer molecular constants (MOLEC IND=2) -------------------------
struct Molec {
  double scor[48][11];   // SCOR(m,iso), 1-based
  double rhoslf[48];     // RHOSLF(m)
  double alfd1[48][11];  // ALFD1(m,iso)
  bool ok[48][11];
};

int molec(const lbl_layer& L, double wtot, Molec& M) {
  // FAD from MOLEC IND=1 (src/oprop.f90:2530-2532)
  double FLN2 = std::log(2.);
  double FAD = FLN2 * 2. * AVOGAD * BOLTZ / (CLIGHT * CLIGHT);
  double RHORAT = (L.pave / P0) * (TEMP0 / L.tave);
  std::memset(&M, 0, sizeof(M));
  for (int m = 1; m <= L.nmol; m++) {
    int nis = LBL_ISO_MAX[m - 1];
    for (int iso = 1; iso <= nis; iso++) {
      double q296, qt;
      // TIPS_2003: scor = Q(296)/Q(T) (src/oprop.f90:6284-6290)
      if (tips_q(m, iso, 296., &q296) && tips_q(m, iso, L.tave, &qt)) {
        M.scor[m][iso] = q296 / qt;
        M.ok[m][iso] = true;
      } else if (m <= LBL_NQMOL) {
        return fail(LBL_E_RANGE, "TIPS temperature out of range");
      }
      M.rhoslf[m] = RHORAT * L.wk[m - 1] / wtot;
      M.alfd1[m][iso] = std::sqrt(FAD * L.tave / LBL_SMASS[m - 1][iso - 1]);
    }
  }
  return LBL_OK;
}

// ---- in-memory TAPE3 ------------------------------------------------------
struct Tape3 {
  const lbl_lines* L;
  std::vector<int64_t> bs;  // block starts, size nb+1
  int64_t nb() const { return (int64_t)bs.size() - 1; }
  explicit Tape3(const lbl_lines* l) : L(l) {
    if (l->nblock > 0 && l->block_start) {
      bs.assign(l->block_start, l->block_start + l->nblock + 1);
    } else {
      for (int64_t s = 0; s < l->n; s += 250) bs.push_back(s);
      bs.push_back(l->n);
    }
  }
  double vmin(int64_t b) const { return L->vnu[bs[b]]; }
  double vmax(int64_t b) const { return L->vnu[bs[b + 1] - 1]; }
};

// Decoded line record as RDLIN/RDLNFL hold it (1-based slot arrays).
struct LineBuf {
  int n = 0;
  double VNU[252], SP[252], ALFA0[252], EPP[252], HWHMS[252], TMPALF[252],
      PSHIFT[252], AMOL[252];
  long MOL[252], IFLG[252];
  double SPPSP[252], RECALF[252], ZETAI[252];
  long IZETA[252];
};

float bits_to_float(int32_t v) {
  float f;
  std::memcpy(&f, &v, 4);
  return f;
}

// Fill a LineBuf from TAPE3 panel b with the O2/N2 width adjustment of
// RDLIN (src/oprop.f90:785-837) / RDLNFL (:3462-3487).
void load_block(const Tape3& t3, int64_t b, LineBuf& B) {
  const lbl_lines* L = t3.L;
  int64_t s = t3.bs[b], e = t3.bs[b + 1];
  B.n = int(e - s);
  for (int i = 1; i <= B.n; i++) {
    int64_t k = s + i - 1;
    B.IFLG[i] = L->iflg[k];
    B.VNU[i] = L->vnu[k];
    B.SP[i] = (double)L->sp[k];
    B.ALFA0[i] = (double)L->alfa[k];
    B.EPP[i] = (double)L->epp[k];
    if (B.IFLG[i] >= 0) {
      B.MOL[i] = L->mol[k];
      B.AMOL[i] = 0.;
    } else {
      B.AMOL[i] = (double)bits_to_float(L->mol[k]);
      B.MOL[i] = 0;
    }
    B.HWHMS[i] = (double)L->hwhms[k];
    B.TMPALF[i] = (double)L->tmpalf[k];
    B.PSHIFT[i] = (double)L->pshift[k];
    long M = B.MOL[i] % 100;
    if (M == 7 && B.IFLG[i] >= 0) {
      double rvmr = 0.21;
      B.ALFA0[i] = (B.ALFA0[i] - rvmr * B.HWHMS[i]) / (1.0 - rvmr);
    }
    if (M == 22 && B.IFLG[i] >= 0) {
      double rvmr = 0.79;
      B.ALFA0[i] = (B.ALFA0[i] - rvmr * B.HWHMS[i]) / (1.0 - rvmr);
    }
  }
}

// ---- shrunk-line TAPE9 ---------------------------------------------------
struct ShrunkBlock {
  double vnulo, vnuhi;
  std::vector<double> VNU, SP, ALFA, EPP, SPP;
  std::vector<long> MOL;
};

// ---- the OPDPTH state -----------------------------------------------------
struct Layer {
  const lbl_run* R;
  const lbl_layer* LY;
  const Tape3* t3;
  const lbl_mtckd* ck;
  int jrad;
  // /FILHDR/
  double PAVE, TAVE, DV, V1, V2, WTOT;
  // far wing /LBLF/
  double V1R4 = 0, V2R4 = 0, DVR4 = 0, BOUND4 = 0;
  long NPTR4 = 0;
  std::vector<double> R4;  // 1-based, 2502+1
  // /ABSORB/
  double V1ABS = 0, V2ABS = 0, DVABS = 0;
  long NPTABS = 0;
  std::vector<double> ABSRB;  // 1-based, 5050+ entries
  int icntnm = 0, ilblf4 = 0;
  std::vector<ShrunkBlock> tape9;
  bool tape9_empty = true;
  Molec mc;
  // stats
  long far_windows = 0;
};

// ---- MT_CKD H2O (mt_ckd_h2o_module.f90:68-296) --------------------------
void myxint(double V1A, double V2A, double DVA, const std::vector<double>& A,
            double AFACT, double VFT, double DVR3, std::vector<double>& R3,
            long N1R3, long N2R3) {
  double RECDVA = 1. / DVA;
  long ILO = fint((V1A + DVA - VFT) / DVR3 + 1. + ONEMI);
  ILO = std::max(ILO, N1R3);
  long IHI = fint((V2A - DVA - VFT) / DVR3 + ONEMI);
  IHI = std::min(IHI, N2R3);
  for (long I = ILO; I <= IHI; I++) {
    double VI = VFT + DVR3 * double(I - 1);
    long J = fint((VI - V1A) * RECDVA + ONEPL);
    double VJ = V1A + DVA * double(J - 1);
    double P = RECDVA * (VI - VJ);
    double C = (3. - 2. * P) * P * P;
    double Bq = 0.5 * P * (1. - P);
    double B1 = Bq * (1. - P);
    double B2 = Bq * P;
    double CONTI = -A[J - 1] * B1 + A[J] * (1. - C + B2) + A[J + 1] * (C + B1) - A[J + 2] * B2;
    R3[I] = R3[I] + CONTI * AFACT;
  }
}

void mt_ckd_h2o(const lbl_mtckd* ck, double p_atm, double t_atm, double h2o_vmr,
                double wv1abs, double wv2abs, double dvabs,
                std::vector<double>& self_absco, std::vector<double>& for_absco,
                bool radflag) {
  // wvn(i) = v0 + (i-1)*dv, i = 1..ncoeffin
  long ncoeffin = ck->n;
  auto wvn = [&](long i) { return ck->v0 + ck->dv * double(i - 1); };
  double dvc = wvn(2) - wvn(1);
  long i = 1;
  while (wvn(i) <= (wv1abs - 2 * dvc)) i++;
  long i1 = i - 1;
  if (i1 == 0) i1 = 1;
  while (wvn(i) < (wv2abs + 2 * dvc)) i++;
  long i2 = i;
  long ncoeff = i2 - i1 + 1;
  double xkt = t_atm / RADCN2;
  double rho_rat = (p_atm / ck->ref_press) * (ck->ref_temp / t_atm);
  // 1-based coefficient arrays with two zero pads for the stencil
  std::vector<double> sh(ncoeff + 4, 0.), fh(ncoeff + 4, 0.), rad(ncoeff + 4, 0.);
  for (long k = 1; k <= ncoeff; k++) {
    long ii = i1 + k - 1;
    sh[k] = ck->self_absco_ref[ii - 1] * std::pow(ck->ref_temp / t_atm, ck->self_texp[ii - 1]);
    sh[k] = sh[k] * h2o_vmr * rho_rat;
    // myradfn (mt_ckd_h2o_module.f90:178-215)
    double xvi = wvn(ii), xviokt = xvi / xkt;
    double r = xvi;
    if (xviokt <= 0.01) r = 0.5 * xviokt * xvi;
    else if (xviokt <= 10.) {
      double e = std::exp(-xviokt);
      r = xvi * (1 - e) / (1. + e);
    }
    rad[k] = r;
    if (radflag) sh[k] = sh[k] * rad[k];
    fh[k] = ck->for_absco_ref[ii - 1] * (1 - h2o_vmr) * rho_rat;
    if (radflag) fh[k] = fh[k] * rad[k];
  }
  long nptabs = fint((wv2abs - wv1abs) / dvabs + 1);
  // pre_xint (mt_ckd_h2o_module.f90:266-296)
  long nbnd_v1c = fint(2 + (wvn(1) - wv1abs) / dvabs + 1.e-5);
  long ist = std::max(1L, nbnd_v1c);
  long nbnd_v2c = fint(1 + (wvn(ncoeffin) - wv1abs) / dvabs + 1.e-5);
  long lst = std::min(nptabs, nbnd_v2c);
  myxint(wvn(i1), wvn(i2), dvc, sh, 1.0, wv1abs, dvabs, self_absco, ist, lst);
  myxint(wvn(i1), wvn(i2), dvc, fh, 1.0, wv1abs, dvabs, for_absco, ist, lst);
}

// The coarse grid of a continuum table (V1S, DVS, NPTS) that FRNCO2,
// o2_ver_1, xn2_r and n2_ver_1 set up alike (src/contnm.f90:1322-1337):
// from one point below V1ABS-DVS to one above V2ABS+DVS.
struct CoarseGrid {
  long I1, NPTC;
  double V1C, V2C, DVC;
};
CoarseGrid coarse_grid(double V1S, double DVS, long NPTS, const Layer& S) {
  CoarseGrid g;
  g.DVC = DVS;
  double V1C = S.V1ABS - g.DVC, V2C = S.V2ABS + g.DVC;
  g.I1 = (V1C < V1S) ? -1 : fint((V1C - V1S) / DVS + 0.01);
  g.V1C = V1S + DVS * double(g.I1 - 1);
  const long I2 = fint((V2C - V1S) / DVS + 0.01);
  g.NPTC = I2 - g.I1 + 3;
  if (g.NPTC > NPTS) g.NPTC = NPTS + 4;
  g.V2C = g.V1C + DVS * double(g.NPTC - 1);
  return g;
}
// pre_xint (:994-1012) and XINT of the coarse values C (1-based) onto ABSRB
void xint_onto_absrb(Layer& S, const CoarseGrid& g, const std::vector<double>& C, double V1SS,
                     double V2SS) {
  const long nbnd_v1c = fint(2 + (V1SS - S.V1ABS) / S.DVABS + 1.e-5);
  const long ist = std::max(1L, nbnd_v1c);
  const long nbnd_v2c = fint(1 + (V2SS - S.V1ABS) / S.DVABS + 1.e-5);
  const long last = std::min(S.NPTABS, nbnd_v2c);
  myxint(g.V1C, g.V2C, g.DVC, C, 1.0, S.V1ABS, S.DVABS, S.ABSRB, ist, last);
}

// CONTNM (src/contnm.f90:199-994): H2O, CO2, the O2 and N2 collision-induced
// bands of the infrared, Rayleigh
void contnm(Layer& S) {
  const lbl_layer& L = *S.LY;
  double RHOAVE = (L.pave / 1013.) * (296. / L.tave);
  double WTOT = L.wbroad;
  for (int m = 1; m <= L.nmol; m++) WTOT = WTOT + L.wk[m - 1];
  double h2o_fac = L.wk[0] / WTOT;
  if ((S.V2 > -20.0) && (S.V1 < 20000.) && ((S.R->xself > 0.) || (S.R->xfrgn > 0))) {
    size_t n = S.ABSRB.size();
    std::vector<double> sh2o(n, 0.), fh2o(n, 0.);
    bool radflag = (S.jrad != 0);
    mt_ckd_h2o(S.ck, L.pave, L.tave, h2o_fac, S.V1ABS, S.V2ABS, S.DVABS, sh2o, fh2o, radflag);
    for (size_t j = 1; j < n; j++) {
      double cself = L.wk[0] * sh2o[j] * S.R->xself;
      double cfor = L.wk[0] * fh2o[j] * S.R->xfrgn;
      S.ABSRB[j] = S.ABSRB[j] + cself + cfor;
    }
  }
  const double XKT = L.tave / RADCN2;
  const double amagat = (L.pave / 1013.) * (273. / L.tave);
  const double x_vmr_h2o = L.wk[0] / WTOT, x_vmr_o2 = L.wk[6] / WTOT;
  const double x_vmr_n2 = 1. - x_vmr_h2o - x_vmr_o2;
  const double wn2 = x_vmr_n2 * WTOT;
  const double xlosmt = 2.68675E+19;
  // CO2 (src/contnm.f90:326-378): FRNCO2's coefficients on its 2 cm-1 grid
  // (:1295-1349, the band-head temperature dependence), the mt_ckd_2.5
  // factors from 2000 to 2998 cm-1, times WCO2, the radiation term when
  // JRAD=1, then XINT onto the ABSRB grid
  if ((S.V2 > -20.0) && (S.V1 < 10000.) && S.R->xco2c > 0.) {
    static const double FCO2T[LBL_FCO2_N] = {LBL_FCO2_VALUES};
    static const double XFACCO2[500] = {LBL_XFACCO2_VALUES};
    static const double TDEP[25] = {LBL_CO2_TDEP_VALUES};
    const double WCO2 = L.wk[1] * RHOAVE * 1.0E-20 * S.R->xco2c;
    const double trat = L.tave / LBL_CO2_TEFF;
    const CoarseGrid g = coarse_grid(LBL_FCO2_V1, LBL_FCO2_DV, LBL_FCO2_N, S);
    std::vector<double> C(g.NPTC + 3, 0.);  // 1-based, zero beyond NPTC
    for (long J = 1; J <= g.NPTC; J++) {
      const long I = g.I1 + (J - 1);
      double fco2 = 0.;
      if (I >= 1 && I <= LBL_FCO2_N) {
        double tcor = 1.;
        if (I >= 1196 && I <= 1220) tcor = std::pow(trat, TDEP[I - 1196]);
        fco2 = tcor * FCO2T[I - 1];
      }
      const double VJ = g.V1C + g.DVC * double(J - 1);
      double CFAC = 1.;
      if (VJ >= 2000. && VJ <= 2998.) {
        const long JFAC = fint((VJ - 1998.) / 2. + 0.00001);
        CFAC = XFACCO2[JFAC - 1];
      }
      fco2 = CFAC * fco2;
      C[J] = fco2 * WCO2;
      if (S.jrad == 1) C[J] = C[J] * RADFN(VJ, XKT);
    }
    xint_onto_absrb(S, g, C, LBL_FCO2_V1, LBL_FCO2_V2);
  }
  // O2 collision-induced fundamental (:491-540, o2_ver_1 :7254-7318)
  if ((S.V2 > 1340.0) && (S.V1 < 1850.) && S.R->xo2cn > 0.) {
    static const double XO2[LBL_O2F_N] = {LBL_O2F_XO2_VALUES};
    static const double XO2T[LBL_O2F_N] = {LBL_O2F_XO2T_VALUES};
    const double tau_fac = S.R->xo2cn * L.wk[6] * 1.e-20 * amagat;
    const double xktfac = (1. / 296.) - (1. / L.tave);
    const double factor = (1.e+20 / xlosmt);
    const CoarseGrid g = coarse_grid(LBL_O2F_V1, LBL_O2F_DV, LBL_O2F_N, S);
    std::vector<double> C(g.NPTC + 3, 0.);
    for (long J = 1; J <= g.NPTC; J++) {
      const long I = g.I1 + (J - 1);
      const double VJ = g.V1C + g.DVC * double(J - 1);
      double c0 = 0.;
      if (I >= 1 && I <= LBL_O2F_N) c0 = factor * XO2[I - 1] * std::exp(XO2T[I - 1] * xktfac) / VJ;
      C[J] = tau_fac * c0;
      if (S.jrad == 1) C[J] = C[J] * RADFN(VJ, XKT);
    }
    xint_onto_absrb(S, g, C, LBL_O2F_V1, LBL_O2F_V2);
  }
  // O2 1.27 um collision-induced band (:543-584, O2INF1 :7384-7440)
  if ((S.V2 > 7536.0) && (S.V1 < 8500.) && S.R->xo2cn > 0.) {
    static const double XO2I1[LBL_O2I1_N] = {LBL_O2I1_X_VALUES};
    const double a_o2 = 1. / 0.446, a_n2 = 0.3 / 0.446, a_h2o = 1.;
    const double tau_fac = S.R->xo2cn * (L.wk[6] / xlosmt) * amagat *
                           (a_o2 * x_vmr_o2 + a_n2 * x_vmr_n2 + a_h2o * x_vmr_h2o);
    const CoarseGrid g = coarse_grid(LBL_O2I1_V1, LBL_O2I1_DV, LBL_O2I1_N, S);
    std::vector<double> C(g.NPTC + 3, 0.);
    for (long J = 1; J <= g.NPTC; J++) {
      const long I = g.I1 + (J - 1);
      const double VJ = g.V1C + g.DVC * double(J - 1);
      double c0 = 0.;
      if (I >= 1 && I <= LBL_O2I1_N) c0 = XO2I1[I - 1] / VJ;
      C[J] = tau_fac * c0;
      if (S.jrad == 1) C[J] = C[J] * RADFN(VJ, XKT);
    }
    xint_onto_absrb(S, g, C, LBL_O2I1_V1, LBL_O2I1_V2);
  }
  // N2 collision-induced rotational band (:745-792, xn2_r :2497-2566)
  if ((S.V2 > -10.0) && (S.V1 < 350.) && S.R->xn2cn > 0.) {
    static const double C296[LBL_N2R296_N] = {LBL_N2R296_C_VALUES};
    static const double SF296[LBL_N2R296_N] = {LBL_N2R296_SF_VALUES};
    static const double C220[LBL_N2R220_N] = {LBL_N2R220_C_VALUES};
    static const double SF220[LBL_N2R220_N] = {LBL_N2R220_SF_VALUES};
    const double tau_fac = S.R->xn2cn * (wn2 / xlosmt) * amagat;
    const double tfac = (L.tave - 296.) / (220. - 296.);
    const CoarseGrid g = coarse_grid(LBL_N2R296_V1, LBL_N2R296_DV, LBL_N2R296_N, S);
    std::vector<double> C(g.NPTC + 3, 0.);
    for (long J = 1; J <= g.NPTC; J++) {
      const long I = g.I1 + (J - 1);
      const double VJ = g.V1C + g.DVC * double(J - 1);
      double c0 = 0., fo2 = 0.;
      if (I >= 1 && I <= LBL_N2R296_N) {
        c0 = C296[I - 1] * std::pow(C220[I - 1] / C296[I - 1], tfac);
        const double sf_T = SF296[I - 1] * std::pow(SF220[I - 1] / SF296[I - 1], tfac);
        fo2 = (sf_T - 1.) * (0.79) / (0.21);
      }
      C[J] = tau_fac * c0 * (x_vmr_n2 + fo2 * x_vmr_o2 + 1. * x_vmr_h2o);
      if (S.jrad == 1) C[J] = C[J] * RADFN(VJ, XKT);
    }
    xint_onto_absrb(S, g, C, LBL_N2R296_V1, LBL_N2R296_V2);
  }
  // N2 collision-induced fundamental (:811-858, n2_ver_1 :2668-2754)
  if ((S.V2 > 2001.77) && (S.V1 < 2897.59) && S.R->xn2cn > 0.) {
    static const double X272[LBL_N2F_N] = {LBL_N2F_X272_VALUES};
    static const double X228[LBL_N2F_N] = {LBL_N2F_X228_VALUES};
    static const double AH2O[LBL_N2F_N] = {LBL_N2F_AH2O_VALUES};
    const double tau_fac = S.R->xn2cn * (wn2 / xlosmt) * amagat;
    const double T = L.tave;
    const double xtfac = ((1. / T) - (1. / 272.)) / ((1. / 228.) - (1. / 272.));
    const double xt_lin = (T - 272.) / (228. - 272.);
    const double a_o2 = 1.294 - 0.4545 * T / 296.;
    const CoarseGrid g = coarse_grid(LBL_N2F_V1, LBL_N2F_DV, LBL_N2F_N, S);
    std::vector<double> C(g.NPTC + 3, 0.);
    for (long J = 1; J <= g.NPTC; J++) {
      const long I = g.I1 + (J - 1);
      const double VJ = g.V1C + g.DVC * double(J - 1);
      double c0 = 0., c1 = 0., c2 = 0.;
      if (I >= 1 && I <= LBL_N2F_N) {
        if (X272[I - 1] > 0. && X228[I - 1] > 0.)
          c0 = X272[I - 1] * std::pow(X228[I - 1] / X272[I - 1], xtfac);
        else
          c0 = X272[I - 1] + (X228[I - 1] - X272[I - 1]) * xt_lin;
        c0 = c0 / VJ;
        c1 = a_o2 * c0;
        c2 = (9. / 7.) * AH2O[I - 1] * c0;
      }
      C[J] = tau_fac * (x_vmr_n2 * c0 + x_vmr_o2 * c1 + x_vmr_h2o * c2);
      if (S.jrad == 1) C[J] = C[J] * RADFN(VJ, XKT);
    }
    xint_onto_absrb(S, g, C, LBL_N2F_V1, LBL_N2F_V2);
  }
  // N2 collision-induced first overtone (:860-906, n2_overtone1 :2916-2968)
  if ((S.V2 > 4340.0) && (S.V1 < 4910.) && S.R->xn2cn > 0.) {
    static const double XN2O[LBL_N2O1_N] = {LBL_N2O1_X_VALUES};
    const double tau_fac = S.R->xn2cn * (wn2 / xlosmt) * amagat *
                           (x_vmr_n2 + 1. * x_vmr_o2 + 1. * x_vmr_h2o);
    const CoarseGrid g = coarse_grid(LBL_N2O1_V1, LBL_N2O1_DV, LBL_N2O1_N, S);
    std::vector<double> C(g.NPTC + 3, 0.);
    for (long J = 1; J <= g.NPTC; J++) {
      const long I = g.I1 + (J - 1);
      const double VJ = g.V1C + g.DVC * double(J - 1);
      double c0 = 0.;
      if (I >= 1 && I <= LBL_N2O1_N) c0 = XN2O[I - 1] / VJ;
      C[J] = tau_fac * c0;
      if (S.jrad == 1) C[J] = C[J] * RADFN(VJ, XKT);
    }
    xint_onto_absrb(S, g, C, LBL_N2O1_V1, LBL_N2O1_V2);
  }
  // Rayleigh extinction (src/contnm.f90:955-976), no aerosols (IAERSL=0)
  if (S.V2 >= 820. && S.R->xrayl > 0.) {
    const double conv_cm2mol = S.R->xrayl * 1.E-20 / (2.68675e-1 * 1.e5);
    const long nptabs = S.NPTABS;  // OPDPTH (src/lblrtm.f90:6222)
    for (long i = 1; i <= nptabs && i < (long)S.ABSRB.size(); i++) {
      double vrayleigh = S.V1ABS + double(i - 1) * S.DVABS;
      double xvrayleigh = vrayleigh / 1.e4;
      double ray_ext = (xvrayleigh * xvrayleigh * xvrayleigh /
                        (9.38076E2 - 10.8426 * (xvrayleigh * xvrayleigh))) *
                       (WTOT * conv_cm2mol);
      if (S.jrad == 1) ray_ext = ray_ext * xvrayleigh;
      else if (S.jrad == 0) ray_ext = ray_ext * xvrayleigh / RADFN(vrayleigh, XKT);
      S.ABSRB[i] = S.ABSRB[i] + ray_ext;
    }
  }
}

// ---- LINF4 + SHRINK (src/oprop.f90:2934-3640) ---------------------------
const double TEMPLC[5] = {0., 200.0, 250.0, 296.0, 340.0};  // 1-based

void shrink(std::vector<double>& VNU, std::vector<double>& SP,
            std::vector<double>& ALFA, std::vector<double>& EPP,
            std::vector<double>& SPP, std::vector<long>& MOL, long& ILO,
            long& IHI, double DVR4) {
  long J = ILO - 1;
  double DV = DVR4 / 2.;
  double VLMT = VNU[ILO] + DV;
  double SUMAL = 0., SUMAD = 0., SUMS = 0., SUMV = 0., SUMC = 0.;
  double SUMAL2 = 0., SUMAD2 = 0., SUMS2 = 0., SUMV2 = 0., SUMC2 = 0.;
  for (long I = ILO; I <= IHI; I++) {
    if (SP[I] < 1.0e-35) {
      SP[I] = 0.0;
      SPP[I] = 0.0;
    }
    if (SPP[I] != 0.0) {
      J = J + 1;
      VNU[J] = VNU[I];
      SP[J] = SP[I];
      ALFA[J] = ALFA[I];
      EPP[J] = EPP[I];
      SPP[J] = SPP[I];
      MOL[J] = MOL[I];
    } else if (MOL[I] != 2) {
      SUMV = SUMV + VNU[I] * SP[I];
      SUMS = SUMS + SP[I];
      SUMAL = SUMAL + SP[I] * ALFA[I];
      SUMAD = SUMAD + SP[I] * EPP[I];
      SUMC = SUMC + SPP[I];
    } else {
      SUMV2 = SUMV2 + VNU[I] * SP[I];
      SUMS2 = SUMS2 + SP[I];
      SUMAL2 = SUMAL2 + SP[I] * ALFA[I];
      SUMAD2 = SUMAD2 + SP[I] * EPP[I];
      SUMC2 = SUMC2 + SPP[I];
    }
    // label 10
    if (I < IHI) {
      if (VNU[I + 1] <= VLMT) continue;
    }
    VLMT = VNU[I] + DV;
    if (SUMS > 0.) {
      J = J + 1;
      SP[J] = SUMS;
      ALFA[J] = SUMAL / SUMS;
      EPP[J] = SUMAD / SUMS;
      VNU[J] = SUMV / SUMS;
      SPP[J] = SUMC;
      MOL[J] = 0;
      SUMAL = SUMAD = SUMS = SUMV = SUMC = 0.;
    }
    if (SUMS2 > 0.) {
      J = J + 1;
      SP[J] = SUMS2;
      ALFA[J] = SUMAL2 / SUMS2;
      EPP[J] = SUMAD2 / SUMS2;
      VNU[J] = SUMV2 / SUMS2;
      MOL[J] = 2;
      SPP[J] = SUMC2;
      SUMAL2 = SUMAD2 = SUMS2 = SUMV2 = SUMC2 = 0.;
    }
  }
  ILO = J + 1;
  IHI = J;
}

int linf4(Layer& S, double V1L4, double V2L4) {
  const lbl_layer& LY = *S.LY;
  const Tape3& t3 = *S.t3;
  const long LIMIN = 1000;
  double VLO = V1L4, VHI = V2L4;
  S.tape9.clear();
  // lnfilhd_4: LINF4 not used if the line file does not intersect V1..V2
  if (t3.nb() == 0 || S.V1 > t3.L->vnu[t3.L->n - 1] || S.V2 < t3.L->vnu[0]) {
    S.tape9_empty = true;
    return LBL_OK;
  }
  S.tape9_empty = false;
  double PAVP0 = S.PAVE / P0;
  double PAVP2 = PAVP0 * PAVP0;
  double TRATIO = S.TAVE / TEMP0;
  double RHORAT = (S.PAVE / P0) * (TEMP0 / S.TAVE);
  double BETA = RADCN2 / S.TAVE;
  double BETA0 = RADCN2 / TEMP0;
  double BETACR = BETA - BETA0;
  const Molec& M = S.mc;
  long ILC;
  for (ILC = 1; ILC <= 4; ILC++)
    if (S.TAVE <= TEMPLC[ILC]) break;
  if (ILC == 1) ILC = 2;
  if (ILC == 5) ILC = 4;
  double RECTLC = 1.0 / (TEMPLC[ILC] - TEMPLC[ILC - 1]);
  double TMPDIF = S.TAVE - TEMPLC[ILC];

  const size_t CAP = 1251 + 260;
  std::vector<double> VNU(CAP), SP(CAP), ALFA(CAP), EPP(CAP), SPP(CAP);
  std::vector<long> MOL(CAP);
  long ILO = 1, IHI = 0, IJ = 0;
  int IEOF = 0;
  int64_t blk = 0;  // next TAPE3 panel for RDLNFL
  LineBuf B;
  auto rdlnfl = [&](std::vector<long>& iout) -> int {
    // RDLNFL: skip panels with VMAX < VLO (src/oprop.f90:3426-3433)
    while (blk < t3.nb() && t3.vmax(blk) < VLO) blk++;
    if (blk >= t3.nb()) return 1;
    load_block(t3, blk, B);
    blk++;
    iout.clear();
    for (int j = 1; j <= B.n; j++)
      if (B.IFLG[j] >= 0) iout.push_back(j);
    return 0;
  };
  std::vector<long> iout;
  while (true) {
    // label 30
    bool goto60 = false;
    int e = rdlnfl(iout);
    if (e >= 1) {
      IEOF = e;
      goto60 = true;
    } else {
      for (size_t jj = 0; jj < iout.size(); jj++) {
        long I = iout[jj];
        long IFLAG = B.IFLG[I];
        double YI = 0., GI = 0., GAMMA1 = 0., GAMMA2 = 0.;
        long m = B.MOL[I] % 100;
        long iso = (B.MOL[I] % 1000) / 100;
        if (m > LBL_MXMOL || m < 1) continue;
        if (iso > LBL_ISO_MAX[m - 1] || iso < 1) continue;
        double SUI = B.SP[I] * LY.wk[m - 1];
        if (SUI == 0.) continue;
        if (B.VNU[I] < VLO) continue;
        IJ = IJ + 1;
        if (IFLAG == 1 || IFLAG == 3) {
          double A[5], Bv[5];
          A[1] = B.VNU[I + 1];
          Bv[1] = B.SP[I + 1];
          A[2] = B.ALFA0[I + 1];
          Bv[2] = B.EPP[I + 1];
          A[3] = B.AMOL[I + 1];
          Bv[3] = B.HWHMS[I + 1];
          A[4] = B.TMPALF[I + 1];
          Bv[4] = B.PSHIFT[I + 1];
          double SLOPEY = (A[ILC] - A[ILC - 1]) * RECTLC;
          double SLOPEG = (Bv[ILC] - Bv[ILC - 1]) * RECTLC;
          if (IFLAG == 1) {
            YI = A[ILC] + SLOPEY * TMPDIF;
            GI = Bv[ILC] + SLOPEG * TMPDIF;
          } else {
            GAMMA1 = A[ILC] + SLOPEY * TMPDIF;
            GAMMA2 = Bv[ILC] + SLOPEG * TMPDIF;
          }
        }
        VNU[IJ] = B.VNU[I] + RHORAT * B.PSHIFT[I];
        ALFA[IJ] = B.ALFA0[I];
        EPP[IJ] = B.EPP[I];
        MOL[IJ] = m;
        if (VNU[IJ] == 0.) SUI = 2. * SUI;
        if (EPP[IJ] <= -1.001) EPP[IJ] = std::fabs(EPP[IJ]);
        if (EPP[IJ] > -0.999)
          SUI = SUI * M.scor[m][iso] * std::exp(-EPP[IJ] * BETACR) *
                (1. + std::exp(-VNU[IJ] * BETA));
        double TMPCOR = std::pow(TRATIO, B.TMPALF[I]);
        double ALFA0I = ALFA[IJ] * TMPCOR;
        double HWHMSI = B.HWHMS[I] * TMPCOR;
        ALFA[IJ] = ALFA0I * (RHORAT - M.rhoslf[m]) + HWHMSI * M.rhoslf[m];
        if (IFLAG == 3) ALFA[IJ] = ALFA[IJ] * (1.0 - GAMMA1 * PAVP0 - GAMMA2 * PAVP2);
        EPP[IJ] = VNU[IJ] * M.alfd1[m][iso];
        SP[IJ] = SUI * (1. + GI * PAVP2);
        SPP[IJ] = SUI * YI * PAVP0;
        if (VNU[IJ] > VHI) {
          IEOF = 1;
          goto60 = true;
          break;
        }
      }
      if (!goto60) {
        if (IJ < LIMIN && IEOF == 0) continue;  // GO TO 30
      }
    }
    // label 60
    IHI = IJ;
    shrink(VNU, SP, ALFA, EPP, SPP, MOL, ILO, IHI, S.DVR4);
    IJ = ILO - 1;
    if (IHI < LIMIN && IEOF == 0) continue;  // GO TO 30
    if (IHI > 0) {
      ShrunkBlock sb;
      sb.vnulo = VNU[1];
      sb.vnuhi = VNU[IHI];
      for (long k = 1; k <= IHI; k++) {
        sb.VNU.push_back(VNU[k]);
        sb.SP.push_back(SP[k]);
        sb.ALFA.push_back(ALFA[k]);
        sb.EPP.push_back(EPP[k]);
        sb.SPP.push_back(SPP[k]);
        sb.MOL.push_back(MOL[k]);
      }
      S.tape9.push_back(std::move(sb));
    }
    if (IEOF == 1) break;
    IJ = 0;
    ILO = 1;
  }
  return LBL_OK;
}

// ---- LBLF4 / RDLIN4 / CONVF4 (src/oprop.f90:3641-4039) ------------------
void convf4(Layer& S, ShrunkBlock& SB, long ILO, long& IHI, double DPTMN,
            double DPTFC) {
  const double ZBND = 64.;
  double RECPI = 1. / (2. * std::asin(1.));
  double ZSQBND = ZBND * ZBND;
  double A3 = (1. + 2. * ZSQBND) / std::pow(1. + ZSQBND, 2);
  double B3 = -1. / std::pow(1. + ZSQBND, 2);
  double VNULST = S.V2R4 + S.BOUND4;
  double BNDSQ = S.BOUND4 * S.BOUND4;
  double r_bndsq = 1. / BNDSQ;
  (void)r_bndsq;
  std::vector<double>& R4 = S.R4;
  for (long I = ILO; I <= IHI; I++) {
    long k = I - 1;  // 0-based into block vectors
    if (SB.SP[k] == 0. && SB.SPP[k] == 0.) continue;
    double ALFADI = SB.EPP[k];
    double ALFALI = SB.ALFA[k];
    double ZETAI = ALFALI / (ALFALI + ALFADI);
    long IZ = fint(100. * ZETAI + ONEPL);
    double ZETDIF = 100. * ZETAI - double(IZ - 1);
    double ALFAVI = (AVRAT(IZ) + ZETDIF * (AVRAT(IZ + 1) - AVRAT(IZ))) * (ALFALI + ALFADI);
    double RALFVI = 1. / ALFAVI;
    double SIL = SB.SP[k] * RECPI * ALFALI;
    double SIV = (ALFALI * RALFVI) * SB.SP[k] * RECPI * RALFVI;
    double SPEAK = A3 * (std::fabs(SIV));
    long JJ = fint((SB.VNU[k] - S.V1R4) / S.DVR4 + 1.);
    JJ = std::max(JJ, 1L);
    JJ = std::min(JJ, S.NPTR4);
    if (SPEAK <= (DPTMN + DPTFC * R4[JJ]) && SB.SPP[k] == 0.) continue;
    double VNUI = SB.VNU[k];
    while (true) {
      // label 30
      double XNUI = VNUI - S.V1R4;
      long JMIN = fint((XNUI - S.BOUND4) / S.DVR4 + 2.);
      if (VNUI >= VNULST) {
        IHI = -1;
        return;
      }
      if (JMIN > S.NPTR4) break;  // GO TO 60
      JMIN = std::max(JMIN, 1L);
      long JMAX = fint((XNUI + S.BOUND4) / S.DVR4 + 1.);
      if (JMAX >= JMIN) {
        JMAX = std::min(JMAX, S.NPTR4);
        double ALFLI2 = ALFALI * ALFALI;
        double ALFVI2 = ALFAVI * ALFAVI;
        double XJJ = double(JMIN - 1) * S.DVR4;
        double F4BND = SIL / (ALFLI2 + BNDSQ);
        double dptrat = SB.SPP[k] / (SB.SP[k] * ALFAVI);
        double rec_alfvi2 = 1. / ALFVI2;
        double siv_a3 = SIV * A3;
        double siv_b3 = SIV * B3;
        if (SB.MOL[k] == 2) {
          for (long J = JMIN; J <= JMAX; J++) {
            double XM = (XJJ - XNUI);
            double XMSQ = XM * XM;
            double ZVSQ = XMSQ * rec_alfvi2;
            double fcnt_fn = (2. - (XMSQ * r_bndsq)) * F4BND;
            double F4FN;
            if (ZVSQ <= ZSQBND) {
              F4FN = (siv_a3 + ZVSQ * siv_b3) - fcnt_fn;
              if (SB.SPP[k] != 0.) F4FN = F4FN + XM * dptrat * F4FN;
            } else {
              F4FN = SIL / (ALFLI2 + XMSQ) - fcnt_fn;
              if (SB.SPP[k] != 0.) F4FN = F4FN + XM * dptrat * F4FN;
            }
            // CHI is identically 1 (chi_fn, src/oprop.f90:4074-4075)
            R4[J] = R4[J] + F4FN;
            XJJ = XJJ + S.DVR4;
          }
        } else {
          for (long J = JMIN; J <= JMAX; J++) {
            double XM = (XJJ - XNUI);
            double XMSQ = XM * XM;
            double ZVSQ = XMSQ * rec_alfvi2;
            double F4FN;
            if (ZVSQ <= ZSQBND) {
              F4FN = (siv_a3 + ZVSQ * siv_b3) - F4BND;
              if (SB.SPP[k] != 0.) F4FN = F4FN + XM * dptrat * F4FN;
            } else {
              F4FN = SIL / (ALFLI2 + XMSQ) - F4BND;
              if (SB.SPP[k] != 0.) F4FN = F4FN + XM * dptrat * F4FN;
            }
            R4[J] = R4[J] + F4FN;
            XJJ = XJJ + S.DVR4;
          }
        }
      }
      // label 50: Van Vleck-Weisskopf image line for 0 < VNU <= 25
      if (VNUI > 0. && VNUI <= 25.) {
        VNUI = -SB.VNU[k];
        SB.SPP[k] = -SB.SPP[k];
        continue;
      }
      break;
    }
  }
}

void lblf4(Layer& S, double V1, double V2) {
  S.far_windows++;
  double DPTMN = S.R->dptmin / RADFN(V2, S.TAVE / RADCN2);
  double DPTFC = S.R->dptfac;
  const long LIMOUT = 2500;
  S.V1R4 = V1;
  S.V2R4 = V2;
  S.NPTR4 = fint((S.V2R4 - S.V1R4) / S.DVR4 + ONEPL);
  S.NPTR4 = std::min(S.NPTR4, LIMOUT);
  S.V2R4 = S.V1R4 + S.DVR4 * double(S.NPTR4 - 1);
  S.R4.assign(2503 + 2, 0.);
  double BETA = RADCN2 / S.TAVE;
  double VLO = S.V1R4 - S.BOUND4;
  double VHI = S.V2R4 + S.BOUND4;
  (void)VHI;
  if (!S.tape9_empty) {
    // RDLIN4 loop: read shrunk blocks from the start, skipping those whose
    // VMAX < VLO; CONVF4 each until IHI=-1 or end of file.
    // (The file copy is modified by the VVW SPP sign flip, as in CONVF4.)
    std::vector<ShrunkBlock> t9 = S.tape9;
    for (size_t b = 0; b < t9.size(); b++) {
      if (t9[b].vnuhi < VLO) continue;
      long IHI = (long)t9[b].VNU.size();
      convf4(S, t9[b], 1, IHI, DPTMN, DPTFC);
      if (IHI == -1) break;
    }
  }
  if (S.jrad == 1) {
    double XKT = 1. / BETA;
    double VITST = S.V1R4 - S.DVR4;
    double RDLAST = -1.;
    long NPTSI1 = 0, NPTSI2 = 0;
    do {
      NPTSI1 = NPTSI2 + 1;
      double VI = S.V1R4 + S.DVR4 * double(NPTSI1 - 1);
      double RDEL;
      double RADVI = RADFNI(VI, S.DVR4, XKT, VITST, RDEL, RDLAST);
      NPTSI2 = fint((VITST - S.V1R4) / S.DVR4 + 0.001);
      NPTSI2 = std::min(NPTSI2, S.NPTR4);
      for (long I = NPTSI1; I <= NPTSI2; I++) {
        S.R4[I] = S.R4[I] * RADVI;
        RADVI = RADVI + RDEL;
      }
    } while (NPTSI2 < S.NPTR4);
  }
}

// ---- XINT, RSYM (src/oprop.f90:2145-2234) -------------------------------
void xint(double V1A, double V2A, double DVA, const double* A, double AFACT,
          double VFT, double DVR3, double* R3, long N1R3, long N2R3) {
  double RECDVA = 1. / DVA;
  long ILO = fint((V1A + DVA - VFT) / DVR3 + 1. + ONEMI);
  ILO = std::max(ILO, N1R3);
  long IHI = fint((V2A - DVA - VFT) / DVR3 + ONEMI);
  IHI = std::min(IHI, N2R3);
  for (long I = ILO; I <= IHI; I++) {
    double VI = VFT + DVR3 * double(I - 1);
    long J = fint((VI - V1A) * RECDVA + ONEPL);
    double VJ = V1A + DVA * double(J - 1);
    double P = RECDVA * (VI - VJ);
    double C = (3. - 2. * P) * P * P;
    double B = 0.5 * P * (1. - P);
    double B1 = B * (1. - P);
    double B2 = B * P;
    double CONTI = -A[J - 1] * B1 + A[J] * (1. - C + B2) + A[J + 1] * (C + B1) - A[J + 2] * B2;
    R3[I] = R3[I] + CONTI * AFACT;
  }
}

void rsym(double* R, double DV, double VFT) {
  long IP = fint((-VFT / DV) + 1. - .000001);
  IP = IP + 1;
  double P = (double(IP - 1) + VFT / DV) * 2.;
  double PST = P;
  if (P > 1.) P = P - 1.;
  double WN1 = -P * (P - 1.) * (P - 2.) / 6.;
  double W0 = (P * P - 1.) * (P - 2.) / 2.;
  double W1 = -P * (P + 1.) * (P - 2.) / 2.;
  double W2 = P * (P * P - 1.) / 6.;
  long K = IP;
  long IPMAX = IP + IP - 1;
  if (PST > 1.) {
    double B1 = R[IP - 2], B2 = R[IP - 1], C1 = R[K], C2;
    for (long I = IP; I <= IPMAX; I++) {
      K = K - 1;
      C2 = C1;
      if (K < 1) return;
      C1 = R[K];
      R[K] = R[K] + WN1 * R[I + 1] + W0 * R[I] + W1 * B2 + W2 * B1;
      B1 = B2;
      B2 = R[I];
      if (K <= 2) continue;
      R[I] = R[I] + WN1 * C2 + W0 * C1 + W1 * R[K - 1] + W2 * R[K - 2];
    }
    return;
  }
  double C1 = R[IP], C2 = R[IP + 1], B2 = R[IP - 1], B1;
  for (long I = IP; I <= IPMAX; I++) {
    K = K - 1;
    B1 = B2;
    B2 = R[I];
    if (K <= 1) return;
    R[I] = R[I] + WN1 * C2 + W0 * C1 + W1 * R[K] + W2 * R[K - 1];
    C2 = C1;
    C1 = R[K];
    R[K] = R[K] + WN1 * R[I + 2] + W0 * R[I + 1] + W1 * B2 + W2 * B1;
  }
}

// Arrays with Fortran lower bounds (RR1(-8704:11169) etc. sized for SAMPLE).
struct FArr {
  std::vector<double> v;
  long lo;
  FArr(long lo_, long hi_) : v(hi_ - lo_ + 1, 0.), lo(lo_) {}
  double& operator[](long i) { return v[i - lo]; }
  double* at1() { return &v[1 - lo] - 1; }  // pointer p with p[i] == (*this)[i]
};

// ---- HIRAC1 (src/oprop.f90:25-633) ---------------------------------------
struct PanelOut {
  double v1p, v2p, dvp;
  long nlim;
  std::vector<double> r;
};

int hirac1(Layer& S, std::vector<PanelOut>& panels) {
  const Shapes& SH = shapes();
  const lbl_run& RN = *S.R;
  const lbl_layer& LY = *S.LY;
  const Tape3& t3 = *S.t3;
  const double DV = S.DV;
  double DPTMN = RN.dptmin;
  if (S.jrad != 1) DPTMN = RN.dptmin / RADFN(S.V2, S.TAVE / RADCN2);
  double DPTFC = RN.dptfac;
  const long NSHIFT = 32;
  double ALFMAX = 4 * RN.sample * DV * 0.04 / RN.alfal0;
  long nALFMAX = fint(ALFMAX / DV);
  long NBOUND = fint((2. * HWF3) * double(nALFMAX) + 0.01);
  const long NLIM1 = 2401, NLIM2 = (NLIM1 / 4) + 1, NLIM3 = (NLIM2 / 4) + 1;
  double DVR2 = (DXF2 / DXF1) * DV;
  double DVR3 = (DXF3 / DXF1) * DV;
  long MAX1 = NSHIFT + NLIM1 + NSHIFT + NBOUND / 2;
  long MAX2 = MAX1 / 4;
  long MAX3 = MAX1 / 16;
  MAX1 = MAX1 + 4 * nALFMAX;
  MAX2 = MAX2 + 16 * nALFMAX / 4 + 1;
  MAX3 = MAX3 + 64 * nALFMAX / 16 + 1;
  double BOUND = double(NBOUND) * DV / 2.;
  long NLO = NSHIFT + 1;
  long NHI = NLIM1 + NSHIFT - 1;
  const long PAD = 4 * MAX1 + 16384;
  FArr R1(-PAD, MAX1 + 64), R2(-PAD, MAX2 + 64), R3(-PAD, MAX3 + 64);
  if (S.ilblf4 == 0) S.R4.assign(2505, 0.);
  double VFT = S.V1 - double(NSHIFT) * DV;
  double VBOT = S.V1 - BOUND;
  double VTOP = S.V2 + BOUND;
  const Molec& M = S.mc;

  double V1R4ST = S.V1R4, V2R4ST = S.V2R4;
  if (S.ilblf4 >= 1) lblf4(S, V1R4ST, V2R4ST);

  // LNCOR1 first-call constants (src/oprop.f90:977-1003)
  double XKT0 = TEMP0 / RADCN2;
  double XKT = S.TAVE / RADCN2;
  double BETACR = (1. / XKT) - (1. / XKT0);
  double TRATIO = S.TAVE / TEMP0;
  double RHORAT = (S.PAVE / P0) * (TEMP0 / S.TAVE);
  double PAVP0 = S.PAVE / P0;
  double PAVP2 = PAVP0 * PAVP0;
  long ILC = 1;
  for (long IL = 1; IL <= 3; IL++) {
    ILC = IL;
    if (S.TAVE < TEMPLC[ILC + 1]) break;
  }
  double RECTLC = 1.0 / (TEMPLC[ILC + 1] - TEMPLC[ILC]);
  double TMPDIF = S.TAVE - TEMPLC[ILC];

  // RDLIN state
  LineBuf B;
  long IOUT[251];
  long ILO = 0, IHI = -999, IDATA = 0;
  int IEOF = 0, IPANEL = 0, ISTOP = 0;
  int64_t blk = 0;
  bool first_read = true;

  auto RDLIN = [&]() -> int {
    if (first_read) {
      blk = 0;
      first_read = false;
    }
    IDATA = 0;
    while (true) {
      if (blk >= t3.nb()) {
        IEOF = 1;
        return LBL_OK;
      }
      if (t3.bs[blk + 1] - t3.bs[blk] > 250) return fail(LBL_E_NREC, "RDLIN; NREC GT LIMIN");
      if (t3.vmax(blk) < VBOT) {
        blk++;
        continue;
      }
      break;
    }
    double VMIN = t3.vmin(blk);
    load_block(t3, blk, B);
    blk++;
    ILO = 1;
    long IJ = 0;
    for (int i = 1; i <= B.n; i++)
      if (B.IFLG[i] >= 0) IOUT[++IJ] = i;
    for (long i = IJ + 1; i <= 250; i++) IOUT[i] = B.n;
    if (VMIN < VBOT) {
      for (long J = 1; J <= IJ; J++) {
        long I = IOUT[J];
        ILO = J;
        if (B.VNU[I] >= VBOT) break;
      }
    }
    for (long J = ILO; J <= IJ; J++) {
      long I = IOUT[J];
      if (B.MOL[I] > 0) {
        IHI = J;
        if (B.VNU[I] > VTOP) break;
      }
    }
    if (IHI < IJ) IDATA = 1;
    return LBL_OK;
  };

  auto LNCOR1 = [&]() {
    for (long J = ILO; J <= IHI; J++) {
      double YI = 0., GI = 0., GAMMA1 = 0., GAMMA2 = 0.;
      long I = IOUT[J];
      long IFLAG = B.IFLG[I];
      long m = B.MOL[I] % 100;
      long iso = (B.MOL[I] % 1000) / 100;
      bool reject = false;
      double SUI = 0.;
      if (m > LBL_MXMOL || m < 1 || iso > LBL_ISO_MAX[m - 1] || iso < 1) {
        reject = true;
      }
      if (!reject) {
        B.MOL[I] = m;
        SUI = B.SP[I] * LY.wk[m - 1];
        if (S.jrad == 1) SUI = SUI * RADFN(B.VNU[I], XKT);
        if (SUI == 0.) reject = true;
      }
      if (!reject) {
        if (IFLAG == 1 || IFLAG == 3) {
          double A[5], Bv[5];
          A[1] = B.VNU[I + 1];
          Bv[1] = B.SP[I + 1];
          A[2] = B.ALFA0[I + 1];
          Bv[2] = B.EPP[I + 1];
          A[3] = B.AMOL[I + 1];
          Bv[3] = B.HWHMS[I + 1];
          A[4] = B.TMPALF[I + 1];
          Bv[4] = B.PSHIFT[I + 1];
          double SLOPEA = (A[ILC + 1] - A[ILC]) * RECTLC;
          double SLOPEB = (Bv[ILC + 1] - Bv[ILC]) * RECTLC;
          if (IFLAG == 1) {
            YI = A[ILC] + SLOPEA * TMPDIF;
            GI = Bv[ILC] + SLOPEB * TMPDIF;
          } else {
            GAMMA1 = A[ILC] + SLOPEA * TMPDIF;
            GAMMA2 = Bv[ILC] + SLOPEB * TMPDIF;
          }
        }
        B.VNU[I] = B.VNU[I] + RHORAT * B.PSHIFT[I];
        double TMPCOR = std::pow(TRATIO, B.TMPALF[I]);
        double ALFA0I = B.ALFA0[I] * TMPCOR;
        double HWHMSI = B.HWHMS[I] * TMPCOR;
        double ALFL = ALFA0I * (RHORAT - M.rhoslf[m]) + HWHMSI * M.rhoslf[m];
        if (IFLAG == 3) ALFL = ALFL * (1.0 - GAMMA1 * PAVP0 - GAMMA2 * PAVP2);
        double ALFAD = B.VNU[I] * M.alfd1[m][iso];
        double ZETA = ALFL / (ALFL + ALFAD);
        B.ZETAI[I] = ZETA;
        double FZETA = 100. * ZETA;
        long IZ = fint(FZETA + ONEPL);
        B.IZETA[I] = IZ;
        double ZETDIF = FZETA - double(IZ - 1);
        double ALFV = (AVRAT(IZ) + ZETDIF * (AVRAT(IZ + 1) - AVRAT(IZ))) * (ALFL + ALFAD);
        if (ALFV < DV) ALFV = DV;
        if (ALFV > ALFMAX) ALFV = ALFMAX;
        if (HWF3 * ALFV + B.VNU[I] < VFT) {
          reject = true;
        } else {
          B.RECALF[I] = 1. / ALFV;
          if (B.EPP[I] <= -1.001) B.EPP[I] = std::fabs(B.EPP[I]);
          if (B.EPP[I] > -0.999)
            SUI = SUI * M.scor[m][iso] * std::exp(-B.EPP[I] * BETACR) *
                  (1. + std::exp(-B.VNU[I] / XKT));
          B.SP[I] = SUI * (1. + GI * PAVP2);
          double SPPI = SUI * YI * PAVP0;
          B.SPPSP[I] = SPPI / B.SP[I];
          if (IFLAG == 0) {
            double SPEAK = SUI * B.RECALF[I];
            if (S.DVR4 <= 0.) {
              if (SPEAK <= DPTMN) reject = true;
            } else {
              long JJ = fint((B.VNU[I] - S.V1R4) / S.DVR4 + 1.);
              JJ = std::max(JJ, 1L);
              JJ = std::min(JJ, S.NPTR4);
              if (SPEAK <= (DPTMN + DPTFC * S.R4[JJ]) && B.SPPSP[I] == 0.) reject = true;
            }
          }
        }
      }
      if (reject) {
        B.SP[I] = 0.;
        B.SPPSP[I] = 0.;
      }
    }
  };

  auto CNVFNV = [&]() {
    const double* F1 = SH.F1;
    const double* F2 = SH.F2;
    const double* F3 = SH.F3;
    const double* FG = SH.FG;
    const double* XVER = SH.XVER;
    double CLC1 = 4. / (double(NX1 - 1));
    double CLC2 = 16. / (double(NX2 - 1));
    double CLC3 = 64. / (double(NX3 - 1));
    double WAVDXF = DV / DXF1;
    double HWDXF = HWF1 / DXF1;
    double CONF2 = DV / DVR2;
    double CONF3 = DV / DVR3;
    long ILAST = ILO - 1;
    if (ILO <= IHI) {
      for (long J = ILO; J <= IHI; J++) {
        long I = IOUT[J];
        if (B.SP[I] == 0.) continue;
        double DEPTHI = B.SP[I] * B.RECALF[I];
        long IZM = B.IZETA[I];
        double ZETDIF = 100. * B.ZETAI[I] - double(IZM - 1);
        double STRF1 = DEPTHI * (CF1(IZM) + ZETDIF * (CF1(IZM + 1) - CF1(IZM)));
        double STRF2 = DEPTHI * (CF2(IZM) + ZETDIF * (CF2(IZM + 1) - CF2(IZM)));
        double STRF3 = DEPTHI * (CF3(IZM) + ZETDIF * (CF3(IZM + 1) - CF3(IZM)));
        double STRD = DEPTHI * (CGAUSS(IZM) + ZETDIF * (CGAUSS(IZM + 1) - CGAUSS(IZM)));
        double STRVER = DEPTHI * (CER(IZM) + ZETDIF * (CER(IZM + 1) - CER(IZM)));
        double ZSLOPE = B.RECALF[I] * WAVDXF;
        double ZINT = (B.VNU[I] - VFT) / DV;
        double BHWDXF = HWDXF / ZSLOPE;
        long JMAX1 = fint(ZINT + BHWDXF + 1.5);
        if (JMAX1 > MAX1) {
          ILAST = J - 1;
          IPANEL = 1;
          ILO = ILAST + 1;
          return;
        }
        long JMIN1 = fint(ZINT - BHWDXF + 1.5);
        double RSHFT = 0.5;
        if (ZINT < 0.0) RSHFT = -RSHFT;
        long J2SHFT = fint(ZINT * (1. - CONF2) + RSHFT);
        long J3SHFT = fint(ZINT * (1. - CONF3) + RSHFT);
        long JMIN2 = JMIN1 - J2SHFT;
        long JMIN3 = JMIN1 - J3SHFT;
        double ZF1L = (double(JMIN1 - 2) - ZINT) * ZSLOPE;
        double ZF2L = (double(JMIN2 - 2) - ZINT * CONF2) * ZSLOPE;
        double ZF3L = (double(JMIN3 - 2) - ZINT * CONF3) * ZSLOPE;
        double ZF1 = ZF1L, ZF2 = ZF2L, ZF3 = ZF3L;
        for (long J1 = JMIN1; J1 <= JMAX1; J1++) {
          long J2 = J1 - J2SHFT;
          long J3 = J1 - J3SHFT;
          ZF3 = ZF3 + ZSLOPE;
          ZF2 = ZF2 + ZSLOPE;
          ZF1 = ZF1 + ZSLOPE;
          long IZ3 = fint(std::fabs(ZF3) + 1.5);
          long IZ2 = fint(std::fabs(ZF2) + 1.5);
          long IZ1 = fint(std::fabs(ZF1) + 1.5);
          R3[J3] = R3[J3] + STRF3 * F3[IZ3];
          R2[J2] = R2[J2] + STRF2 * F2[IZ2];
          R1[J1] = R1[J1] + STRF1 * F1[IZ1] + STRD * FG[IZ1] + STRVER * XVER[IZ1];
        }
        if (B.SPPSP[I] != 0.) {
          double DPTRAT = B.SPPSP[I];
          STRF3 = STRF3 * CLC3 * DPTRAT;
          STRF2 = STRF2 * CLC2 * DPTRAT;
          STRF1 = STRF1 * CLC1 * DPTRAT;
          STRD = STRD * CLC1 * DPTRAT;
          STRVER = STRVER * CLC1 * DPTRAT;
          for (long J1 = JMIN1; J1 <= JMAX1; J1++) {
            long J2 = J1 - J2SHFT;
            long J3 = J1 - J3SHFT;
            ZF3L = ZF3L + ZSLOPE;
            ZF2L = ZF2L + ZSLOPE;
            ZF1L = ZF1L + ZSLOPE;
            long IZ3 = fint(std::fabs(ZF3L) + 1.5);
            long IZ2 = fint(std::fabs(ZF2L) + 1.5);
            long IZ1 = fint(std::fabs(ZF1L) + 1.5);
            R3[J3] = R3[J3] + STRF3 * F3[IZ3] * ZF3L;
            R2[J2] = R2[J2] + STRF2 * F2[IZ2] * ZF2L;
            R1[J1] = R1[J1] + (STRF1 * F1[IZ1] + STRD * FG[IZ1] + STRVER * XVER[IZ1]) * ZF1L;
          }
        }
      }
      ILAST = IHI;
      IPANEL = (int)IDATA;
    } else {
      IPANEL = 1;
    }
    ILO = ILAST + 1;
  };

  long N1R1 = 1, N2R1, N1R2 = 1, N2R2, N1R3 = 1, N2R3;
  (void)N1R1;
  int IFPAN = 1;
  double XKTP = S.TAVE / RADCN2;

  auto PANEL = [&]() {
    const double X00 = -7. / 128., X01 = 105. / 128., X02 = 35. / 128., X03 = -5. / 128.,
                 X10 = -1. / 16., X11 = 9. / 16.;
    double DVP = DV;
    ISTOP = 0;
    double V2P;
    if ((VFT + double(NHI - 1) * DVP) > S.V2) {
      NHI = fint((S.V2 - VFT) / DVP + 1.);
      V2P = VFT + double(NHI - 1) * DVP;
      if (V2P < S.V2) {
        V2P = V2P + DVP;
        NHI = NHI + 1;
      }
      ISTOP = 1;
    } else {
      V2P = VFT + double(NHI - 1) * DV;
    }
    long NLIM = NHI - NLO + 1;
    double V1P = VFT + double(NLO - 1) * DV;
    long LIMLO = N1R2;
    if (N1R2 == 1) LIMLO = LIMLO + 4;
    long LIMHI = (NHI / 4) + 1;
    long J = LIMLO, J3 = 0;
    for (J = LIMLO; J <= LIMHI; J += 4) {
      J3 = (J - 1) / 4 + 1;
      R2[J] = R2[J] + R3[J3];
      R2[J + 1] = R2[J + 1] + X00 * R3[J3 - 1] + X01 * R3[J3] + X02 * R3[J3 + 1] + X03 * R3[J3 + 2];
      R2[J + 2] = R2[J + 2] + X10 * (R3[J3 - 1] + R3[J3 + 2]) + X11 * (R3[J3] + R3[J3 + 1]);
      R2[J + 3] = R2[J + 3] + X03 * R3[J3 - 1] + X02 * R3[J3] + X01 * R3[J3 + 1] + X00 * R3[J3 + 2];
    }
    if (LIMLO <= LIMHI && ISTOP == 1) {
      J3 = J3 + 1;
      R2[J] = R2[J] + R3[J3];
      R2[J + 1] = R2[J + 1] + X00 * R3[J3 - 1] + X01 * R3[J3] + X02 * R3[J3 + 1] + X03 * R3[J3 + 2];
    }
    for (long Jr = NLO; Jr <= NHI; Jr += 4) {
      long J2 = (Jr - 1) / 4 + 1;
      R1[Jr] = R1[Jr] + R2[J2];
      R1[Jr + 1] = R1[Jr + 1] + X00 * R2[J2 - 1] + X01 * R2[J2] + X02 * R2[J2 + 1] + X03 * R2[J2 + 2];
      R1[Jr + 2] = R1[Jr + 2] + X10 * (R2[J2 - 1] + R2[J2 + 2]) + X11 * (R2[J2] + R2[J2 + 1]);
      R1[Jr + 3] = R1[Jr + 3] + X03 * R2[J2 - 1] + X02 * R2[J2] + X01 * R2[J2 + 1] + X00 * R2[J2 + 2];
    }
    if (S.jrad == 0) {
      double VI = V1P - DV;
      double VITST = VI;
      double RDLAST = -1.;
      long NPTSI1 = NLO - 1, NPTSI2 = NLO - 1;
      do {
        NPTSI1 = NPTSI2 + 1;
        VI = VFT + double(NPTSI1 - 1) * DV;
        double RDEL;
        double RADVI = RADFNI(VI, DV, XKTP, VITST, RDEL, RDLAST);
        NPTSI2 = fint((VITST - VFT) / DV + 0.001);
        NPTSI2 = std::min(NPTSI2, NHI);
        for (long I = NPTSI1; I <= NPTSI2; I++) {
          R1[I] = R1[I] * RADVI;
          RADVI = RADVI + RDEL;
        }
      } while (NPTSI2 < NHI);
    }
    PanelOut po;
    po.v1p = V1P;
    po.v2p = V2P;
    po.dvp = DVP;
    po.nlim = NLIM;
    po.r.resize(NLIM);
    for (long k = 0; k < NLIM; k++) po.r[k] = R1[NLO + k];
    panels.push_back(std::move(po));
    VFT = VFT + double(NLIM1 - 1) * DV;
    if (ISTOP != 1) {
      for (long Jj = NLIM1; Jj <= MAX1; Jj++) R1[Jj - NLIM1 + 1] = R1[Jj];
      for (long Jj = MAX1 - NLIM1 + 2; Jj <= MAX1; Jj++) R1[Jj] = 0.;
      for (long Jj = NLIM2; Jj <= MAX2; Jj++) R2[Jj - NLIM2 + 1] = R2[Jj];
      for (long Jj = MAX2 - NLIM2 + 2; Jj <= MAX2; Jj++) R2[Jj] = 0.;
      for (long Jj = NLIM3; Jj <= MAX3; Jj++) R3[Jj - NLIM3 + 1] = R3[Jj];
      for (long Jj = MAX3 - NLIM3 + 2; Jj <= MAX3; Jj++) R3[Jj] = 0.;
      NLO = NSHIFT + 1;
    }
  };

  // ---- panel loop (src/oprop.f90:444-542) ----
  enum { L60, L70, L80 } st = L60;
  while (true) {
    if (st == L60) {
      if (IEOF != 0) {
        st = L80;
        continue;
      }
      int rc = RDLIN();
      if (rc != LBL_OK) return rc;
      if (IEOF != 0) {
        st = L80;
        continue;
      }
      LNCOR1();
      st = L70;
    }
    if (st == L70) {
      CNVFNV();
      if (IPANEL == 0) {
        st = L60;
        continue;
      }
      st = L80;
    }
    // label 80
    if (IFPAN == 1) {
      IFPAN = 0;
      N1R1 = 1;
      N1R2 = 1;
      N1R3 = 1;
    } else {
      N1R1 = NSHIFT + 1;
      N1R2 = (NSHIFT / 4) + 1 + 4;
      N1R3 = (NSHIFT / 16) + 1 + 3;
    }
    N2R1 = NLIM1 + NSHIFT - 1;
    N2R2 = NLIM2 + (NSHIFT / 4) - 1 + 4;
    N2R3 = NLIM3 + (NSHIFT / 16) - 1 + 3;
    (void)N2R1;
    (void)N2R2;
    if (VFT <= 0. && g_rsym) {
      rsym(R1.at1(), DV, VFT);
      rsym(R2.at1(), DVR2, VFT);
      rsym(R3.at1(), DVR3, VFT);
    }
    if (S.ilblf4 >= 1) xint(S.V1R4, S.V2R4, S.DVR4, S.R4.data(), 1.0, VFT, DVR3, R3.at1(), N1R3, N2R3);
    if (S.icntnm >= 1)
      xint(S.V1ABS, S.V2ABS, S.DVABS, S.ABSRB.data(), 1., VFT, DVR3, R3.at1(), N1R3, N2R3);
    PANEL();
    if (ISTOP != 1) {
      if (S.ilblf4 >= 1) {
        double VF1 = VFT - 2. * S.DVR4;
        VF1 = S.V1 + std::floor((VF1 - S.V1) / S.DVR4) * S.DVR4;
        double VF2 = VFT + 2. * S.DVR4 + double(N2R3 + 4) * DVR3;
        if (VF2 > S.V2R4 && S.V2R4 != V2R4ST) lblf4(S, VF1, V2R4ST);
      }
      st = L70;
      continue;
    }
    break;
  }
  return LBL_OK;
}

// ---- OPDPTH (src/lblrtm.f90:6135-6287) -----------------------------------
int opdpth(const lbl_run* run, const lbl_layer* ly, const Tape3& t3,
           const lbl_mtckd* ck, int* jrad, std::vector<PanelOut>& panels) {
  Layer S;
  S.R = run;
  S.LY = ly;
  S.t3 = &t3;
  S.ck = ck;
  S.jrad = *jrad;
  S.PAVE = ly->pave;
  S.TAVE = ly->tave;
  S.DV = ly->dv;
  S.V1 = run->v1;
  S.V2 = run->v2;
  S.WTOT = ly->wbroad;
  for (int m = 0; m < ly->nmol; m++) S.WTOT += ly->wk[m];
  S.icntnm = run->icntnm;
  S.ilblf4 = run->ilblf4;
  if (ly->nmol < 1 || ly->nmol > LBL_NQMOL)
    return fail(LBL_E_RANGE, "nmol outside the tabulated TIPS molecules 1-7");
  int rc = molec(*ly, S.WTOT, S.mc);
  if (rc != LBL_OK) return rc;
  double XKT = S.TAVE / RADCN2;
  if (((S.V1 / XKT) < 5.) && (S.jrad != -1)) S.jrad = 0;
  S.DVABS = 0.;
  S.ABSRB.assign(5050 + 8, 0.);
  if (S.icntnm != 0) {
    if (!ck) return fail(LBL_E_NOTREADY, "continuum table missing");
    S.DVABS = 1.;
    S.V1ABS = (double)fint(S.V1);
    if (S.V1 < 0.) S.V1ABS = S.V1ABS - 1.;
    S.V1ABS = S.V1ABS - 3. * S.DVABS;
    S.V2ABS = (double)fint(S.V2 + 3. * S.DVABS + 0.5);
    S.NPTABS = fint((S.V2ABS - S.V1ABS) / S.DVABS + 1.5);
    contnm(S);
  }
  S.DVR4 = 0.;
  if (S.ilblf4 >= 1) {
    double ALFAV = run->sample * S.DV;
    double ALFAV4 = 64. * ALFAV;
    S.DVR4 = ALFAV4 / run->sample;
    S.BOUND4 = 25.;
    if (S.ilblf4 == 2 && S.PAVE <= 0.5) S.BOUND4 = 5.;
    S.V1R4 = S.V1 - 2. * S.DVR4;
    S.V2R4 = S.V2 + 2. * S.DVR4;
    double V1L4 = S.V1R4 - S.BOUND4 - S.DVR4;
    double V2L4 = S.V2R4 + S.BOUND4 + 2 * S.DVR4;
    rc = linf4(S, V1L4, V2L4);
    if (rc != LBL_OK) return rc;
  }
  rc = hirac1(S, panels);
  *jrad = S.jrad;
  return rc;
}

// ---- merge (src/xmerge.f90) ----------------------------------------------
double PLANCK(double VI, double XKT) {
  double VPLANCK = 0.;
  if (XKT > 0.0) {
    double VKT = XKT;
    double VIOKT = VI / VKT;
    if (VIOKT < 1e-2) {
      VPLANCK = (VI * VI) * VKT / (1. + 0.5 * VIOKT);
    } else if (VIOKT <= 80.) {
      double VEXPNEG = std::exp(-VIOKT);
      VPLANCK = (VI * VI * VI) * VEXPNEG / (1. - VEXPNEG);
    }
  }
  return VPLANCK * RADCN1;
}

// EMIN, LTE branch with XKTB<=0 and IAERSL=0 (src/xmerge.f90:1795-1855)
// With XKTB > 0 (the symmetric tangent path, IPATHL=2, and specular
// reflection, src/xmerge.f90:1980-2019) also the emission EMB of the
// layer's other crossing, with the other level's temperature.
void emin(const PanelOut& p, double XKT, double XKTA, std::vector<double>& EM,
          std::vector<double>& TR, double XKTB = 0., std::vector<double>* EMB = nullptr) {
  long NLIM = p.nlim;
  EM.assign(NLIM + 1, 0.);
  TR.assign(NLIM + 1, 0.);
  if (EMB) EMB->assign(NLIM + 1, 0.);
  double rec_6 = 1. / 6.;
  double VI = p.v1p;
  double bb_dif = 0., bb_dif_b = 0.;
  for (long I = 1; I <= NLIM; I++) {
    double BB = PLANCK(VI, XKT);
    if (XKTA > 0.) bb_dif = PLANCK(VI, XKTA) - BB;
    if (EMB && XKTB > 0.) bb_dif_b = PLANCK(VI, XKTB) - BB;
    double ODVI = p.r[I - 1];
    if (ODVI < -OD_LO) ODVI = -OD_LO;
    double tr_i = std::exp(-ODVI);
    double f_i;
    if (ODVI <= OD_LO) f_i = rec_6 * ODVI;
    else f_i = 1. - 2. * (tr_i / (tr_i - 1.) + 1. / ODVI);
    TR[I] = tr_i;
    const double abs_i = 1. - tr_i;
    EM[I] = abs_i * (BB + bb_dif * f_i);
    if (EMB) (*EMB)[I] = abs_i * (BB + bb_dif_b * f_i);
    VI = VI + p.dvp;
  }
}

struct MPanel {
  double v1p, v2p, dvp;
  long nlim;
  std::vector<double> rad, tr;
};

// XKTA of EMINIT/RADMRG (src/xmerge.f90:2405-2424): the upper level's
// temperature looking down (IPATHL=1), the lower level's looking up (3).
double xkta_of(const lbl_run& R, const lbl_layer& L) {
  return (R.ipathl == 3 ? L.tzl : L.tzu) / RADCN2;
}

// The reflected atmosphere (IPATHL=-1): looking down with a boundary
// reflectivity, EMINIT/RADMRG turn IPATHL=1 into -1 (src/xmerge.f90:2389,
// 2725; IBPROP=1 when BNDRFL is non-zero, src/lblrtm.f90:979-980), specular
// (SURF_REFL 's'), constant BNDRFL(1).
bool reflected(const lbl_run& R) { return R.ipathl == 1 && R.bndrfl != 0.; }

// EMINIT (src/xmerge.f90:2436-2484): IPATHL=1 with the surface term when
// TBND>0; IPATHL=3 with no boundary at the first layer (XMERGE :136-141).
void eminit(const lbl_run& R, const lbl_layer& L, const std::vector<PanelOut>& od,
            std::vector<MPanel>& out) {
  double XKT = L.tave / RADCN2;
  double TBND = (R.ipathl == 1) ? R.tmpbnd : 0.;
  double XKTBND = TBND / RADCN2;
  double XKTA = xkta_of(R, L);
  out.clear();
  for (const PanelOut& p : od) {
    std::vector<double> EM, TR, EMB;
    const bool tangent = R.ipathl == 2, refl = reflected(R);
    emin(p, XKT, XKTA, EM, TR, (tangent || refl) ? L.tzl / RADCN2 : 0.,
         (tangent || refl) ? &EMB : nullptr);
    MPanel mp{p.v1p, p.v2p, p.dvp, p.nlim, {}, {}};
    mp.rad.resize(p.nlim);
    mp.tr.resize(p.nlim);
    if (refl) {
      // IPATHL=-1 (:2486-2540, constant EMISIV and REFLCT): the layer's
      // downward emission reflected at the surface, and the surface's own
      double EMISIV = R.bndemi, REFLCT = R.bndrfl;
      double VI = p.v1p;
      for (long J = 1; J <= p.nlim; J++) {
        double BB = PLANCK(VI, XKTBND);
        EM[J] = EM[J] + EMB[J] * REFLCT * TR[J] + TR[J] * BB * EMISIV;
        VI = VI + p.dvp;
      }
    } else if (tangent) {
      // IPATHL=2, IANT=0 (:2442-2447): the tangent layer crossed twice
      for (long J = 1; J <= p.nlim; J++) {
        const double TRJ = TR[J];
        EM[J] = EM[J] + EMB[J] * TRJ;
        TR[J] = TR[J] * TRJ;
      }
    } else if (TBND > 0.) {
      double EMISIV = R.bndemi;
      double VI = p.v1p;
      for (long J = 1; J <= p.nlim; J++) {
        double BB = PLANCK(VI, XKTBND);
        EM[J] = EM[J] + TR[J] * BB * EMISIV;
        VI = VI + p.dvp;
      }
    }
    for (long J = 1; J <= p.nlim; J++) {
      mp.rad[J - 1] = EM[J];
      mp.tr[J - 1] = TR[J];
    }
    out.push_back(std::move(mp));
  }
}

// RADMRG + RADNN, IPATHL=1 (src/xmerge.f90:2587-2895, 2899-3130)
// The RADMRG/RADNN panel loop with the layer's (EM, TR) supplied per panel
// by `layer`: EMIN for the forward merge; the analytic-Jacobian rows use the
// same loop to regrid a field onto the layer grid (EM = 0, TR = 1) and to
// carry a row through the layer (EM = 0, TR = the layer transmittance).
int radmrg_core(const lbl_run& R, const lbl_layer& L, double DVL,
                const std::vector<MPanel>& old, const std::vector<PanelOut>& od,
                const std::function<void(size_t, const PanelOut&, std::vector<double>&,
                                         std::vector<double>&)>& layer,
                std::vector<MPanel>& out, const std::vector<double>* EMBp = nullptr) {
  double DVK = L.dv;
  long ITYPE;
  if (DVL == DVK) ITYPE = 0;
  else if (DVL > DVK) ITYPE = fint(DVK / (DVL - DVK) + 0.5);
  else ITYPE = -fint(DVL / (DVK - DVL) + 0.5);
  if (ITYPE < 0) return fail(LBL_E_ITYPE, " RADMRG; ITYPE LT 0 ");
  double XKT = L.tave / RADCN2;
  double XKTA = xkta_of(R, L);
  const bool down = R.ipathl == 3;  // IPATH_FLG = 3
  // IPATH_FLG = 2 (the symmetric tangent path): the layer's other crossing,
  // EMB (filled by `layer` with EM and TR), seen through the old path
  const bool tangent = R.ipathl == 2 && EMBp != nullptr;
  // IPATH_FLG = -10 (the reflected atmosphere, specular): EMB goes down
  // through the old path, is reflected and comes back up through it
  const bool refl = reflected(R) && EMBp != nullptr;
  const double REFLCT = R.bndrfl;
  double ATYPE = ITYPE;
  long LL = ITYPE + 1;
  double AP = 1.0 / (ATYPE + 1.0);
  double A1[12] = {0}, A2[12] = {0}, A3[12] = {0}, A4[12] = {0};
  for (long JPG = 1; JPG <= ITYPE; JPG++) {
    double APG = JPG;
    long IPL = JPG + 1;
    double P = 1.0 - (AP * APG);
    A1[IPL] = -P * (P - 1.0) * (P - 2.0) / 6.0;
    A2[IPL] = (P * P - 1.0) * (P - 2.0) * 0.5;
    A3[IPL] = -P * (P + 1.0) * (P - 2.0) * 0.5;
    A4[IPL] = P * (P * P - 1.0) / 6.0;
  }
  std::vector<double> RADO(5000 + 20, 0.), TRAO(5000 + 20, 0.);
  long NPE = 0;
  double V2PO = 0., DVPO = 0.;
  size_t oi = 0;  // next old panel
  out.clear();
  (void)XKT;
  (void)XKTA;
  for (size_t pi = 0; pi < od.size(); pi++) {
    const PanelOut& p = od[pi];
    std::vector<double> EM, TR;
    layer(pi, p, EM, TR);
    if (V2PO <= p.v2p + DVPO) {
      while (true) {
        if (oi >= old.size()) break;
        const MPanel& op = old[oi++];
        V2PO = op.v2p;
        DVPO = op.dvp;
        for (long k = 0; k < op.nlim; k++) {
          RADO[NPE + 1 + k] = op.rad[k];
          TRAO[NPE + 1 + k] = op.tr[k];
        }
        NPE = op.nlim + NPE;
        if (!(V2PO <= p.v2p + DVPO)) break;
      }
    }
    if (RADO[0] == 0.0 && TRAO[0] == 0.0) {
      RADO[0] = RADO[1];
      TRAO[0] = TRAO[1];
    }
    if (V2PO + DVPO >= R.v2) {
      RADO[NPE + 1] = RADO[NPE];
      RADO[NPE + 2] = RADO[NPE];
      TRAO[NPE + 1] = TRAO[NPE];
      TRAO[NPE + 2] = TRAO[NPE];
    }
    long NPL = 1;
    // RADNN, IPATH_FLG = 1 (upwelling) or 3 (downwelling,
    // src/xmerge.f90:2989-2995, 3007-3013, 3117-3130, 3150-3166)
    long NLIM = p.nlim;
    long LLM1 = std::max(LL - 1, 1L);
    long IPL = 0;
    for (long NL = 1; NL <= LL; NL++) {
      IPL = (NPL + NL - 1) - LLM1;
      if (NL > 1) IPL = IPL - 1;
      if (NL == 1) {
        for (long I = NL; I <= NLIM; I += LL) {
          IPL = IPL + LLM1;
          if (refl) {
            // :3051-3066
            const double TRTEMP = TR[I] * TRAO[IPL];
            EM[I] = TR[I] * RADO[IPL] + EM[I] + (*EMBp)[I] * TRAO[IPL] * TRTEMP * REFLCT;
            TR[I] = TRTEMP;
            continue;
          }
          if (tangent) {
            // :2997-3005
            const double TRTEMP = TR[I] * TRAO[IPL];
            EM[I] = TR[I] * RADO[IPL] + EM[I] + (*EMBp)[I] * TRTEMP;
            TR[I] = TR[I] * TRTEMP;
            continue;
          }
          if (down) EM[I] = RADO[IPL] + EM[I] * TRAO[IPL];
          else EM[I] = TR[I] * RADO[IPL] + EM[I];
          TR[I] = TR[I] * TRAO[IPL];
        }
      } else {
        double A1N = A1[NL], A2N = A2[NL], A3N = A3[NL], A4N = A4[NL];
        for (long I = NL; I <= NLIM; I += LL) {
          IPL = IPL + LLM1;
          if (refl) {
            // :3197-3215
            const double TRAOI = A1N * TRAO[IPL - 1] + A2N * TRAO[IPL] + A3N * TRAO[IPL + 1] +
                                 A4N * TRAO[IPL + 2];
            const double TRTEMP = TR[I] * TRAOI;
            EM[I] = TR[I] * (A1N * RADO[IPL - 1] + A2N * RADO[IPL] + A3N * RADO[IPL + 1] +
                             A4N * RADO[IPL + 2]) +
                    EM[I] + (*EMBp)[I] * TRAOI * TRTEMP * REFLCT;
            TR[I] = TRTEMP;
            continue;
          }
          if (tangent) {
            // :3132-3148
            const double TRTEMP = TR[I] * (A1N * TRAO[IPL - 1] + A2N * TRAO[IPL] +
                                           A3N * TRAO[IPL + 1] + A4N * TRAO[IPL + 2]);
            EM[I] = TR[I] * (A1N * RADO[IPL - 1] + A2N * RADO[IPL] + A3N * RADO[IPL + 1] +
                             A4N * RADO[IPL + 2]) +
                    EM[I] + (*EMBp)[I] * TRTEMP;
            TR[I] = TR[I] * TRTEMP;
            continue;
          }
          if (down) {
            double TRAOI = A1N * TRAO[IPL - 1] + A2N * TRAO[IPL] + A3N * TRAO[IPL + 1] +
                           A4N * TRAO[IPL + 2];
            EM[I] = A1N * RADO[IPL - 1] + A2N * RADO[IPL] + A3N * RADO[IPL + 1] +
                    A4N * RADO[IPL + 2] + EM[I] * TRAOI;
            TR[I] = TR[I] * TRAOI;
          } else {
            EM[I] = TR[I] * (A1N * RADO[IPL - 1] + A2N * RADO[IPL] + A3N * RADO[IPL + 1] +
                             A4N * RADO[IPL + 2]) +
                    EM[I];
            TR[I] = TR[I] * (A1N * TRAO[IPL - 1] + A2N * TRAO[IPL] + A3N * TRAO[IPL + 1] +
                             A4N * TRAO[IPL + 2]);
          }
        }
      }
    }
    NPL = IPL;
    MPanel mp{p.v1p, p.v2p, p.dvp, p.nlim, {}, {}};
    mp.rad.assign(EM.begin() + 1, EM.end());
    mp.tr.assign(TR.begin() + 1, TR.end());
    out.push_back(std::move(mp));
    long IPLn = -1;
    for (long NL = NPL; NL <= NPE; NL++) {
      IPLn = IPLn + 1;
      RADO[IPLn] = RADO[NL];
      TRAO[IPLn] = TRAO[NL];
    }
    NPE = IPLn;
  }
  return LBL_OK;
}

int radmrg(const lbl_run& R, const lbl_layer& L, double DVL,
           const std::vector<MPanel>& old, const std::vector<PanelOut>& od,
           std::vector<MPanel>& out) {
  const double XKT = L.tave / RADCN2, XKTA = xkta_of(R, L);
  // IPATHL=2 and -1: XKTB the lower level's temperature (:2765-2773)
  const bool tangent = R.ipathl == 2 || reflected(R);
  const double XKTB = tangent ? L.tzl / RADCN2 : 0.;
  std::vector<double> EMB;
  return radmrg_core(R, L, DVL, old, od,
                     [&](size_t, const PanelOut& p, std::vector<double>& EM,
                         std::vector<double>& TR) {
                       emin(p, XKT, XKTA, EM, TR, XKTB, tangent ? &EMB : nullptr);
                     },
                     out, tangent ? &EMB : nullptr);
}

// EMBND (src/xmerge.f90:3652-3733) with a constant emissivity (BNDEMI(1);
// BNDEMI(2:3) = 0): the boundary beyond the last layer seen through the
// whole path, R += T * EMISIV * B(TBND); XMERGE applies it at the last layer
// looking up (IPATHL=3, :140, 157).
void embnd(const lbl_run& R, std::vector<MPanel>& acc) {
  const double TBND = R.tmpbnd;
  if (!(TBND > 0.)) return;
  const double XKTBND = TBND / RADCN2;
  for (MPanel& p : acc) {
    double VI = p.v1p;
    for (long J = 0; J < p.nlim; J++) {
      double BB = PLANCK(VI, XKTBND);
      p.rad[J] = p.rad[J] + p.tr[J] * R.bndemi * BB;
      VI = VI + p.dvp;
    }
  }
}

// ABSMRG (src/xmerge.f90:437-682): optical-depth sum with 4-point regrid.
int absmrg(const lbl_layer& L, double DVL, const std::vector<MPanel>& old,
           const std::vector<PanelOut>& od, std::vector<MPanel>& out) {
  double DVK = L.dv;
  long ITYPE = 0;
  if (DVL == DVK) ITYPE = 0;
  if (DVL > DVK) ITYPE = fint(DVK / (DVL - DVK) + 0.5);
  if (DVL < DVK) ITYPE = -fint(DVL / (DVK - DVL) + 0.5);
  if (ITYPE < 0) return fail(LBL_E_ITYPE, " ABSMRG: ITYPE LT 0 ");
  out.clear();
  double FACT = 1.;
  size_t oi = 0, ki = 0;
  std::vector<double> OLDR1(2410 + 8, 0.), R1(2410 + 8, 0.);
  double V1PO = 0, DVPO = 0;
  long NLIMO = 0;
  auto read_old = [&](long at) -> bool {
    if (oi >= old.size()) return false;
    const MPanel& op = old[oi++];
    V1PO = op.v1p;
    DVPO = op.dvp;
    NLIMO = op.nlim;
    for (long k = 0; k < NLIMO; k++) OLDR1[at + k] = op.rad[k];
    return true;
  };
  double V1P = 0, V2P = 0, DVP = 0;
  long NLIM = 0;
  auto read_new = [&]() -> bool {
    if (ki >= od.size()) return false;
    const PanelOut& p = od[ki++];
    V1P = p.v1p;
    V2P = p.v2p;
    DVP = p.dvp;
    NLIM = p.nlim;
    for (long k = 0; k < NLIM; k++) R1[1 + k] = p.r[k];
    return true;
  };
  auto emit = [&]() {
    MPanel mp{V1P, V2P, DVP, NLIM, {}, {}};
    mp.rad.assign(R1.begin() + 1, R1.begin() + 1 + NLIM);
    mp.tr.assign(NLIM, 0.);
    out.push_back(std::move(mp));
  };
  if (ITYPE == 0) {
    while (true) {
      read_old(1);
      if (!read_new()) break;
      for (long k = 1; k <= NLIM; k++) R1[k] = R1[k] + OLDR1[k];
      emit();
    }
    return LBL_OK;
  }
  double A1[12], A2[12], A3[12], A4[12], SAVOR1[6] = {0};
  double ATYPE = ITYPE;
  double AP = 1.0 / (ATYPE + 1.0);
  long LL = ITYPE + 1;
  for (long JPG = 1; JPG <= ITYPE; JPG++) {
    double APG = JPG;
    double P = 1.0 - (AP * APG);
    A1[JPG] = -P * (P - 1.0) * (P - 2.0) / 6.0;
    A2[JPG] = (P * P - 1.0) * (P - 2.0) * 0.5;
    A3[JPG] = -P * (P + 1.0) * (P - 2.0) * 0.5;
    A4[JPG] = P * (P * P - 1.0) / 6.0;
  }
  read_old(1);
  long MAXLF = NLIMO;
  long NVS = 1;
  if (!read_new()) return LBL_OK;
  long II = 1;
  double DIF = DVP * 0.01;
  // align the first points (labels 100-120)
  if (!(std::fabs(V1PO - V1P) < DIF)) {
    double V1PN;
    while (true) {
      NVS = NVS + 1;
      V1PN = V1PO + DVPO * (NVS - 1);
      if (std::fabs(V1PN - V1P) < DIF) break;
      if (V1PN < V1P) continue;
      bool found = false;
      while (true) {
        II = II + 1;
        double V1PP = V1P + DVP * (II - 1);
        if (std::fabs(V1PN - V1PP) < DIF) {
          found = true;
          break;
        }
        if (V1PP < V1PN) continue;
        break;
      }
      if (found) break;
    }
  }
  R1[II] = FACT * R1[II] + OLDR1[NVS];
  II = II + 1;
  while (true) {
    // label 130
    long JJ = 1;
    for (long JPG = 1; JPG <= LL; JPG++) {
      bool at210 = false;
      if (JPG == LL) {
        R1[II] = R1[II] + OLDR1[NVS];
      } else {
        double OLDR1Y;
        if (NVS == 1) OLDR1Y = (SAVOR1[4] == 0.0) ? OLDR1[1] : SAVOR1[4];
        else OLDR1Y = OLDR1[NVS - 1];
        double OLDR1I = A1[JJ] * OLDR1Y + A2[JJ] * OLDR1[NVS] + A3[JJ] * OLDR1[NVS + 1] +
                        A4[JJ] * OLDR1[NVS + 2];
        R1[II] = R1[II] + OLDR1I;
      }
      // label 190
      NVS = NVS + 1;
      if (!(NVS <= MAXLF - 2)) {
        SAVOR1[1] = OLDR1[NVS - 1];
        SAVOR1[2] = OLDR1[NVS];
        SAVOR1[3] = OLDR1[NVS + 1];
        SAVOR1[4] = OLDR1[NVS - 2];
        if (read_old(4)) {
          MAXLF = NLIMO + 3;
          OLDR1[1] = SAVOR1[1];
          OLDR1[2] = SAVOR1[2];
          OLDR1[3] = SAVOR1[3];
          NVS = 2;
        } else {
          at210 = true;
        }
      }
      if (at210) {
        II = II + 1;
        double AVRG = (SAVOR1[3] + SAVOR1[2]) * 0.5;
        while (II <= NLIM) {
          R1[II] = FACT * R1[II] + AVRG;
          II = II + 1;
        }
        emit();
        if (!read_new()) return LBL_OK;
        II = 1;
        continue;  // next JPG (Fortran falls to 240)
      }
      // label 200
      II = II + 1;
      JJ = JJ + 1;
      if (II > NLIM) {
        emit();
        if (!read_new()) return LBL_OK;
        II = 1;
      }
    }
    NVS = NVS - 1;
  }
}

std::vector<PanelOut> panels_from_array(const lbl_run& R, double dv, const double* a,
                                        int64_t n) {
  // the PANEL output sequence of OPDPTH for a layer of spacing dv
  std::vector<PanelOut> ps;
  double VFT = R.v1 - 32. * dv;
  int64_t off = 0;
  while (off < n) {
    long NHI = 2432, NLO = 33;
    double V2P;
    bool last = false;
    if ((VFT + double(NHI - 1) * dv) > R.v2) {
      NHI = fint((R.v2 - VFT) / dv + 1.);
      V2P = VFT + double(NHI - 1) * dv;
      if (V2P < R.v2) {
        V2P = V2P + dv;
        NHI = NHI + 1;
      }
      last = true;
    } else {
      V2P = VFT + double(NHI - 1) * dv;
    }
    PanelOut p;
    p.nlim = NHI - NLO + 1;
    p.v1p = VFT + double(NLO - 1) * dv;
    p.v2p = V2P;
    p.dvp = dv;
    p.r.assign(a + off, a + std::min<int64_t>(n, off + p.nlim));
    p.r.resize(p.nlim, 0.);
    off += p.nlim;
    ps.push_back(std::move(p));
    VFT = VFT + 2400. * dv;
    if (last) break;
  }
  return ps;
}

int64_t npts_of(const lbl_run& R, double dv) {
  double VFT = R.v1 - 32. * dv;
  int64_t n = 0;
  while (true) {
    long NHI = 2432;
    if ((VFT + double(NHI - 1) * dv) > R.v2) {
      NHI = fint((R.v2 - VFT) / dv + 1.);
      double V2P = VFT + double(NHI - 1) * dv;
      if (V2P < R.v2) NHI = NHI + 1;
      return n + (NHI - 33 + 1);
    }
    n += 2400;
    VFT = VFT + double(2401 - 1) * dv;
  }
}

// ---- PNLINT (src/oprop.f90:1564-1806) -----------------------------------
// The layer optical depth streamed through PANEL's 2400-point panels
// (src/oprop.f90:1435-1451, 1524-1555) and re-gridded to DVOUT as PNLINT
// does: the SAVEd V1PO/NLIM1, the 2400-point output panels (R1OUT), the
// four cases at label 20, the A1..A4 weights at P=0.01*JP.  R1 here is the
// panel passed as R1(NLO): R1(-2..0) hold the previous panel's last points
// (PANEL's shift keeps NSHIFT=32 of them), R1(1..NLIM) the panel, and
// R1(NLIM+1..NLIM+2) the next panel's first points -- which PNLINT reads
// only with zero weight (JP=0) except in the last panel, where they are the
// two padded copies of R1(NLIM).
struct Pnlint {
  double DVOUT;
  double V1PO = 0., V1PO_SAVE = 0.;
  long NLIM1 = 1;
  double A1[101], A2[101], A3[101], A4[101];
  std::vector<double> out;
  explicit Pnlint(double dvout) : DVOUT(dvout) {
    for (int JP = 0; JP <= 100; JP++) {
      double APG = JP, P = 0.01 * APG;
      A1[JP] = -P * (P - 1.0) * (P - 2.0) / 6.0;
      A2[JP] = (P * P - 1.0) * (P - 2.0) * 0.5;
      A3[JP] = -P * (P + 1.0) * (P - 2.0) * 0.5;
      A4[JP] = P * (P * P - 1.0) / 6.0;
    }
  }
  // One call: R1 points to R1(1) of a buffer valid from R1(-2) to R1(NLIM+2).
  void call(double* R1, long NLIM, double V1P, double V2P, double DVP, double V2, int ISTOP) {
    if (V1PO_SAVE != 0.0) V1PO = V1PO_SAVE;
    int NPPANL = 1;
    double ATYPE = 9.999E09;
    if (DVP == DVOUT) ATYPE = 0.;
    if (DVOUT > DVP) ATYPE = DVP / (DVOUT - DVP) + 0.5;
    if (DVOUT < DVP) ATYPE = -DVOUT / (DVP - DVOUT) - 0.5;
    if (std::fabs(DVOUT - DVP) < 1.E-8) ATYPE = 0.;
    if (ATYPE == 0.) {
      for (long i = 1; i <= NLIM; i++) out.push_back(R1[i - 1]);
      V1PO_SAVE = V1PO;
      return;
    }
    auto r1 = [&](long j) -> double& { return R1[j - 1]; };
    if (V1PO == 0.0) {
      r1(-1) = r1(1);
      r1(0) = r1(1);
      V1PO = V1P;
      NLIM1 = 1;
    }
    if (ISTOP == 1) {
      r1(NLIM + 1) = r1(NLIM);
      r1(NLIM + 2) = r1(NLIM);
      NLIM = NLIM + 2;
      V2P = V2P + 2. * DVP;
    }
    const long LIMOUT = 2400;
    double R1OUT[2401];
    int ILAST = 0;
    double V2PO;
    long NLIM2;
    for (;;) {  // label 20
      V2PO = V1PO + double(LIMOUT) * DVOUT;
      if (V2P <= V2PO + DVP && ILAST == 0 && NPPANL <= 0) break;
      if ((V1PO + double(LIMOUT - 1) * DVOUT) > V2) {
        NLIM2 = fint((V2 - V1PO) / DVOUT + 1.);
        V2PO = V1PO + double(NLIM2 - 1) * DVOUT;
        if (V2PO < V2) {
          V2PO = V2PO + DVOUT;
          NLIM2 = NLIM2 + 1;
        }
        ILAST = 1;
        if (ISTOP != 1 && V2PO > V2P - DVP) {
          NLIM2 = fint(((V2P - DVP - V1PO) / DVOUT) + 1.);
          V2PO = V1PO + double(NLIM2 - 1) * DVOUT;
          if (V2PO + DVOUT < V2P - DVP) {
            NLIM2 = NLIM2 + 1;
            V2PO = V2PO + DVOUT;
          }
          ILAST = 0;
        }
      } else {
        NLIM2 = LIMOUT;
        V2PO = V1PO + double(NLIM2 - 1) * DVOUT;
        if (V2PO > V2P - DVP) {
          NLIM2 = fint(((V2P - DVP - V1PO) / DVOUT) + 1.);
          V2PO = V1PO + double(NLIM2 - 1) * DVOUT;
          if (V2PO + DVOUT < V2P - DVP) {
            NLIM2 = NLIM2 + 1;
            V2PO = V2PO + DVOUT;
          }
        }
        ILAST = 0;
      }
      const double RATDV = DVOUT / DVP;
      const double FJ1DIF = (V1PO - V1P) / DVP + 1. + 2.;
      for (long II = NLIM1; II <= NLIM2; II++) {  // label 30
        double FJJ = FJ1DIF + RATDV * double(II - 1);
        long JJ = fint(FJJ) - 2;
        long JP = fint((FJJ - double(JJ)) * 100. - 199.5);
        JP = JP < 0 ? 0 : (JP > 100 ? 100 : JP);
        R1OUT[II] = A1[JP] * r1(JJ - 1) + A2[JP] * r1(JJ) + A3[JP] * r1(JJ + 1) +
                    A4[JP] * r1(JJ + 2);
      }
      if (NLIM2 == LIMOUT || ILAST == 1) {
        for (long i = 1; i <= NLIM2; i++) out.push_back(R1OUT[i]);
        NLIM1 = 1;
        NPPANL = 0;
        V1PO = V2PO + DVOUT;
        if ((V1PO + double(LIMOUT) * DVOUT) > (V2P - DVP)) NPPANL = 1;
      } else {
        NLIM1 = NLIM2 + 1;
        NPPANL = -1;
      }
      if (ILAST == 1) break;
    }
    if (ILAST == 1) {
      V1PO = 0.0;
      NPPANL = 1;
    }
    V1PO_SAVE = V1PO;
  }
};

// PANEL's panel geometry around PNLINT for a layer OD on V1 + i*DV.
int pnlint_layer(const lbl_run& R, double DV, double DVOUT, const double* od, int64_t n,
                 std::vector<double>* res) {
  if (!(DVOUT > 0.) || !(DV > 0.)) return fail(LBL_E_ARG, "DV and DVOUT must be positive");
  if (DVOUT > DV && !(std::fabs(DVOUT - DV) < 1.E-8))
    return fail(LBL_E_ARG, "DVOUT MUST BE < DV");
  if (npts_of(R, DV) != n) return fail(LBL_E_ARG, "n_in does not match the layer grid");
  Pnlint S(DVOUT);
  double VFT = R.v1 - 32. * DV;
  const long NLO = 33;
  std::vector<double> buf(2432 + 8);
  int64_t g0 = 0;
  for (;;) {
    long NHI = 2432;
    int ISTOP = 0;
    double V2P;
    if ((VFT + double(NHI - 1) * DV) > R.v2) {
      NHI = fint((R.v2 - VFT) / DV + 1.);
      V2P = VFT + double(NHI - 1) * DV;
      if (V2P < R.v2) {
        V2P = V2P + DV;
        NHI = NHI + 1;
      }
      ISTOP = 1;
    } else {
      V2P = VFT + double(NHI - 1) * DV;
    }
    const long NLIM = NHI - NLO + 1;
    const double V1P = VFT + double(NLO - 1) * DV;
    // buf[3 + j - 1] = R1(j), j = -2 .. NLIM+2
    double* R1 = buf.data() + 3;
    for (long j = -2; j <= NLIM + 2; j++) {
      int64_t g = g0 + j - 1;
      R1[j - 1] = (g >= 0 && g < n) ? od[g] : 0.;
    }
    S.call(R1, NLIM, V1P, V2P, DV, R.v2, ISTOP);
    if (ISTOP) break;
    VFT = VFT + double(2401 - 1) * DV;
    g0 += 2400;
  }
  *res = std::move(S.out);
  return LBL_OK;
}

// ---- SCANFN (src/postsub.f90:25-560) -------------------------------------
// The scanning functions on the global output grid: the tabulated shapes
// (SHAPET :1377-1400, SHAPEG src/oprop.f90:1912-1942, SINCSQ :2445-2484,
// SINC :2486-2525), SHRKSC's compression (:1276-1376: the largest ratio of
// JRATIO not above HWHM/12/DVI, group means), CONVSC's sums (:1516-1598: each
// compressed input spread over its JMIN..JMAX with XF(|ZF|+1.5)), PANLSC's
// last point (:1600-1660).  ZPEAK and ZF are taken from one global origin
// (the reference's panel origins and incremental ZF round slightly
// differently).
struct ScanOracle {
  int jfn = 0;
  double hwhm = 0, sample = 0, dvo = 0, hwf = 0, dxf = 0, bound = 0, vft0 = 0, vbot = 0, vtop = 0;
  long nf = 0, nfmax = 0, nnhi = 0;
  double bfov = 0;         // JFN 5/6: the field-of-view half angle, radians
  double dvint = 0;        // SCANFN's DVINT: a coarser input is interpolated first
  std::vector<double> xf;  // 1-based
};

int scan_setup(const lbl_scan& sc, double dv_in, ScanOracle& S) {
  static const double HWJ[7] = {1., 2., 4., 54.1826, 119.332818, 1., 1.};
  static const double DXJ[7] = {0., 0.02, 0.02, 0.02, 0.02, 0., 0.};
  static const long NJ[7] = {0, 101, 201, 2710, 5968, 0, 0};
  static const long NJMX[7] = {0, 251, 251, 2760, 6018, 0, 0};
  static const double SMPLJ[7] = {.5, 2., 4., 4., 4., .5, .5};
  static const double XSCAL[7] = {0., 0., 0., 1.391557377, 1.89549425, 0., 0.};
  const double PI = 2. * std::asin(1.);
  double HWHM = sc.hwhm;
  int JFN = sc.jfn;
  if (!(HWHM > 0.) || !(sc.v2 > sc.v1) || !(dv_in > 0.)) return fail(LBL_E_ARG, "scan: HWHM, V1, V2, DV");
  if (JFN < 0) {
    JFN = -JFN;
    if (JFN != 3 && JFN != 4) return fail(LBL_E_ARG, "SCANFN; INVALID JFN");
  }
  if (JFN < 0 || JFN > 6)
    return fail(LBL_E_ARG, "scan: JFN 0-6 (rectangle, triangle, Gauss, sinc^2, sinc, FOV boxes)");
  const double XSCALE = XSCAL[JFN];
  if (sc.jfn < 0) HWHM = HWHM / (PI / XSCALE);
  S.jfn = JFN;
  S.hwf = HWJ[JFN];
  S.dxf = DXJ[JFN];
  S.nf = NJ[JFN];
  S.nfmax = NJMX[JFN];
  double SAMPLE = SMPLJ[JFN];
  if (sc.sampl < 0.) SAMPLE = HWHM / (-sc.sampl);
  else if (sc.sampl > 0.) SAMPLE = sc.sampl;
  // DVINT (:245-265)
  double DVINT = HWHM / 12.;
  if (JFN == 5 || JFN == 6) DVINT = sc.v1 * std::pow(HWHM * 3.141592654 / 180., 2) / 24;
  S.dvint = DVINT;
  if (dv_in > DVINT) return fail(LBL_E_RANGE, "scan: input DV above DVINT (interpolate first)");
  S.hwhm = HWHM;
  S.sample = SAMPLE;
  S.dvo = HWHM / SAMPLE;
  if (JFN == 5 || JFN == 6) {
    // CNVVRC / CNVVRL: boxes at V1 + (NB-1) DVO up to V2, no IRATIO
    S.bfov = HWHM * 3.141592654 / 180.;
    long NB = 1;
    while (sc.v1 + double(NB) * S.dvo <= sc.v2) NB++;
    S.nnhi = NB + 32;
    return LBL_OK;
  }
  if (JFN == 0) {
    // adjacent boxes of 2 HWHM (SCANFN :393-399): DVO a whole number of DVI
    const long IRATIO = fint(S.dvo / dv_in + 0.5);
    S.dvo = double(IRATIO) * dv_in;
    if (IRATIO < 2) return fail(LBL_E_RANGE, "scan: IRATIO LESS THAN 2, NO SCANFN");
    long NB = 1;
    while (sc.v1 + double(NB) * S.dvo <= sc.v2) NB++;
    S.nnhi = NB + 32;  // boxes NB = 1.. with VCNT <= V2
    return LBL_OK;
  }
  const long NBOUND = fint((2. * S.hwf) * SAMPLE + 0.01);
  S.bound = double(NBOUND) * S.dvo / 2.;
  S.vft0 = sc.v1 - 32. * S.dvo;
  S.vbot = sc.v1 - S.bound;
  S.vtop = sc.v2 + S.bound;
  S.nnhi = fint((sc.v2 - S.vft0) / S.dvo + 1.5);
  // the shape table
  S.xf.assign(S.nfmax + 2, 0.);
  std::vector<double>& XF = S.xf;
  if (JFN == 1) {
    XF[1] = 0.5;
    for (long I = 2; I <= S.nf; I++) {
      double X = double(I - 1) * S.dxf;
      XF[I] = 0.5 * (1. - 0.5 * X);
    }
  } else if (JFN == 2) {
    const double FLN2 = std::log(2.), RECPI = 1. / (2. * std::asin(1.));
    const double FGNORM = std::sqrt(FLN2 * RECPI);
    XF[1] = FGNORM * std::exp(-FLN2 * 0.);
    for (long JJ = 2; JJ <= S.nf; JJ++) {
      double X = double(JJ - 1) * S.dxf;
      double XSQ = X * X;
      XF[JJ] = FGNORM * std::exp(-FLN2 * XSQ);
    }
    XF[S.nf] = 0.;
  } else {
    const double XNORM = XSCALE / PI;
    XF[1] = XNORM;
    for (long I = 2; I <= S.nf; I++) {
      double X = double(I - 1) * S.dxf;
      double A = X * XSCALE;
      double sx = std::sin(A) / A;
      XF[I] = (JFN == 3) ? XNORM * (sx * sx) : XNORM * sx;
    }
  }
  return LBL_OK;
}

// SCNINT (src/postsub.f90:824-1035) with INTERP (:2940-3215, I4PT=1): the
// spectrum, read in 2400-point panels (RDPANL :2768-2870, no conversion),
// onto DVO = DVINT from V1 to V1 + NUM DVO, NUM = (V2-V1)/DVO + 0.5, by the
// 4-point cubic whose weights are tabulated at 201 values of the fraction P
// (C1..C4 :2990-3001); P is carried from point to point by adding
// DVO/DVI and restarted from the wavenumber at each output panel (2400
// points) and whenever the input panel runs out.
int scnint(const double* spec, long n, double v1_in, double dv_in, double DVO,
           std::vector<double>& out) {
  const long NUMCOF = 201;
  const double XNUMCF = double(NUMCOF);
  double C1[203], C2[203], C3[203], C4[203];
  for (long IP = 0; IP <= NUMCOF + 1; IP++) {
    const double P = (double(IP) - 1.0) / (XNUMCF - 1.0);
    const double PP = P * P;
    C1[IP] = -P / 2.0 * ((1 - P) * (1 - P));
    C2[IP] = 1.0 - PP * (3.0 - 2.0 * P) + PP / 2.0 * (1.0 - P);
    C3[IP] = PP * (3.0 - 2.0 * P) + P / 2.0 * ((1.0 - P) * (1.0 - P));
    C4[IP] = -PP / 2 * (1.0 - P);
  }
  const double V1 = v1_in;
  long NUM = fint(((v1_in + double(n - 1) * dv_in - V1) / DVO) + 0.5);
  const double V2 = V1 + double(NUM) * DVO;
  out.clear();
  std::vector<double> T(2410 + 8, 0.), R(2401 + 8, 0.);
  // RDPANL: panel k, its points into T(5..), VMIN = V1P - 4 DVI, NNI = NLIMP + 4
  long k = 0;
  double V1I = 0., V2I = 0.;
  const double DVI = dv_in;
  long NNI = 0;
  bool eof = false;
  auto rdpanl = [&]() {
    const long a = 2400 * k;
    if (a >= n) {
      eof = true;
      return;
    }
    const long m = std::min(2400L, n - a);
    const double V1P = v1_in + double(a) * dv_in, V2P = v1_in + double(a + m - 1) * dv_in;
    for (long i = 0; i < m; i++) T[5 + i] = spec[a + i];
    V1I = V1P - 4.0 * DVI;
    V2I = V2P;
    NNI = m + 4;
    k++;
  };
  for (long II = 1; II <= 4; II++) T[II] = 0.0;
  rdpanl();
  if (eof) return fail(LBL_E_ARG, "SCNINT: empty spectrum");
  double V1J = V1;
  const double DVJ = DVO;
  const double VRATIO = DVJ / DVI;
  double VJ = V1J;
  T[4] = 2.0 * T[5] - T[6];
  long J1 = 0, J2 = 0;
  auto otpanl = [&](long NNJ) {
    for (long J = 1; J <= NNJ; J++) out.push_back(R[J]);
  };
  while (V1J < V1I) {  // label 20: output points below the input
    J1 = 1;
    J2 = std::min(fint((V1I - V1J) / DVJ) + 1, 2400L);
    for (long J = J1; J <= J2; J++) R[J] = 0.0;
    const double V2J = V1J + DVJ * double(J2 - 1);
    otpanl(J2);
    V1J = V2J + DVJ;
    VJ = V1J;
  }
  long guard = 0;
  for (;;) {  // label 40
    if (++guard > 100000000L) return fail(LBL_E_ARG, "SCNINT: no progress");
    long I = fint((VJ - V1I) / DVI + 1.00001);
    const double VI = V1I + DVI * double(I - 1);
    double P = (VJ - VI) / DVI;
    J1 = fint((VJ - V1J) / DVJ + 1.001);
    J2 = std::min(std::min(fint((V2 - V1J) / DVJ + 1.001), fint((V2I - DVI - V1J) / DVJ + 1.)),
                  2400L);
    for (long J = J1; J <= J2; J++) {
      const long IP = fint(P * XNUMCF + 1.00001);
      R[J] = C1[IP] * T[I - 1] + C2[IP] * T[I] + C3[IP] * T[I + 1] + C4[IP] * T[I + 2];
      P = P + VRATIO;
      if (P >= 1.0) {
        I = fint(double(I) + P);
        P = P - double(fint(P));
      }
    }
    VJ = V1J + DVJ * double(J2);
    if (J2 >= 2400 || VJ >= V2) {
      const double V2J = V1J + DVJ * double(J2 - 1);
      otpanl(J2);
      V1J = V2J + DVJ;
      J2 = 0;
    }
    if (VJ >= V2) break;
    if (eof) {  // label 80: zeros to V2
      for (;;) {
        J1 = J2 + 1;
        J2 = std::min(fint((V2 - V1J) / DVJ + 1.0001), 2400L);
        for (long J = J1; J <= J2; J++) R[J] = 0.0;
        VJ = V1J + DVJ * double(J2);
        if (J2 >= 2400 || VJ >= V2) {
          const double V2J = V1J + DVJ * double(J2 - 1);
          otpanl(J2);
          V1J = V2J + DVJ;
          J2 = 0;
        }
        if (!(VJ < V2)) break;
      }
      break;
    }
    if (I >= NNI - 2) {
      for (long II = 1; II <= 4; II++) T[II] = T[II + NNI - 4];
      rdpanl();
      if (eof) {
        T[NNI + 1] = 2.0 * T[NNI] - T[NNI - 1];
        T[NNI + 2] = 0.0;
        V2I = V2I + DVI;
      }
    }
  }
  return LBL_OK;
}

int orc_scnint_impl(const double* spec, long n, double v1_in, double dv_in, double dvo,
                    std::vector<double>& out) {
  return scnint(spec, n, v1_in, dv_in, dvo, out);
}

int scan_spectrum(const lbl_scan& sc, const double* spec, int64_t n, double v1_in, double dv_in,
                  std::vector<double>& out) {
  ScanOracle S;
  int rc = scan_setup(sc, dv_in, S);
  if (rc == LBL_E_RANGE && dv_in > S.dvint && S.dvint > 0.) {
    // SCANFN :322-345: a spectrum coarser than DVINT is first interpolated
    std::vector<double> fine;
    rc = scnint(spec, (long)n, v1_in, dv_in, S.dvint, fine);
    if (rc) return rc;
    return scan_spectrum(sc, fine.data(), (int64_t)fine.size(), v1_in, S.dvint, out);
  }
  if (rc) return rc;
  // RDSCAN (:1411-1514): JEMIT=-1 convolves the absorption 1 - S
  std::vector<double> s(spec, spec + n);
  if (sc.jabs) for (auto& x : s) x = 1. - x;
  if (S.jfn == 0 || S.jfn == 5 || S.jfn == 6) {
    // CNVRCT (:1779-1985), CNVVRC (:1986-2214), CNVVRL (:2216-2440) on the
    // whole input: box NB at V1 + (NB-1) DVO, centred with half width HWHM
    // (JFN 0), centred from VCNT (1 - BFOV^2/4) to VCNT (1 + BFOV^2/4) (5),
    // from VLFT to VLFT (1 + BFOV^2/2) (6); inner points weight 1, the end
    // points the fraction of their interval inside the box; the weighted mean
    const double DVI = dv_in, V1I = v1_in;
    const long NNI = (long)n;
    const double BFOV = S.bfov;
    auto edges = [&](long NB, double& VLFT, double& VRGT) {
      const double V0 = sc.v1 + double(NB - 1) * S.dvo;
      if (S.jfn == 5) {
        VLFT = V0 * (1 - BFOV * BFOV / 4);
        VRGT = V0 * (1 + BFOV * BFOV / 4);
      } else if (S.jfn == 6) {
        VLFT = V0;
        VRGT = V0 * (1 + BFOV * BFOV / 2);
      } else {
        VLFT = V0 - S.hwhm;
        VRGT = V0 + S.hwhm;
      }
    };
    // the boxes must lie inside the spectrum (the reference outputs no box
    // that runs past its data)
    double vfirst, vdum, vlast;
    edges(1, vfirst, vdum);
    edges(S.nnhi - 32, vdum, vlast);
    if (v1_in > vfirst - DVI || v1_in + double(n - 1) * DVI < vlast + DVI)
      return fail(LBL_E_RANGE, "scan: the boxes must lie inside the spectrum");
    out.clear();
    for (long NB = 1; NB <= S.nnhi - 32; NB++) {
      double VLFT, VRGT;
      edges(NB, VLFT, VRGT);
      const double RL = (VLFT - V1I) / DVI + 1, RR = (VRGT - V1I) / DVI + 1;
      long IL = fint(RL + 0.5), IH = fint(RR + 0.5);
      double WGTL = ((V1I + double(IL - 1) * DVI) + DVI / 2. - VLFT) / DVI;
      double WGTR = (VRGT - ((V1I + double(IH - 1) * DVI) - DVI / 2.)) / DVI;
      long NEP = 2;
      if (IH > NNI) {
        IH = NNI;
        WGTR = 1.;
        if (IL == IH) {
          WGTR = 0.;
          NEP = 1;
        }
      }
      if (IL <= 1) {
        IL = 1;
        WGTL = 1.;
        if (IL >= IH) {
          WGTL = 0.;
          NEP = 1;
        }
      }
      double SUMJ = 0.;
      for (long I = IL + 1; I <= IH - 1; I++) SUMJ = SUMJ + s[I - 1];
      SUMJ = SUMJ + s[IL - 1] * WGTL;
      SUMJ = SUMJ + s[IH - 1] * WGTR;
      const double RNJ = double(IH - IL + 1 - NEP) + WGTL + WGTR;
      out.push_back(SUMJ / RNJ);
    }
    return LBL_OK;
  }
  // SHRKSC
  static const long JRATIO[25] = {0, 1, 2, 3, 4, 5, 6, 8, 10, 12, 15, 16, 20,
                                  24, 25, 30, 32, 40, 48, 50, 60, 75, 80, 100, 120};
  double DVI = dv_in;
  double DVSC = S.hwhm / 12.;
  long IRATSH = fint(DVSC / DVI + 0.5);
  for (int I = 2; I <= 24; I++)
    if (JRATIO[I] > IRATSH) {
      IRATSH = JRATIO[I - 1];
      break;
    }
  if (IRATSH > JRATIO[24]) IRATSH = JRATIO[24];
  double V1SHFT = 0.;
  if (IRATSH > 1) {
    DVSC = double(IRATSH) * DVI;
    V1SHFT = double(IRATSH - 1) * DVI / 2.;
  } else {
    IRATSH = 1;
    DVSC = DVI;
  }
  const double SRATIO = IRATSH;
  const int64_t nc = n / IRATSH;
  std::vector<double> sc1(nc + 1, 0.);  // 1-based
  for (int64_t k = 1; k <= nc; k++) {
    double SUMK = 0.;
    for (long j = 0; j < IRATSH; j++) SUMK = SUMK + s[(k - 1) * IRATSH + j];
    sc1[k] = SUMK / SRATIO;
  }
  const double V1I = v1_in + V1SHFT;
  // CONVSC on the global output grid (R1(1) at VFT0)
  const double RATIO = DVSC / S.dvo, DVODX = S.dvo / S.dxf, HWBND = S.hwf / S.dvo;
  const double ZINT = (V1I - S.vft0) / S.dvo;
  const double ZSLOPE = DVODX / S.hwhm, ZBOUND = HWBND * S.hwhm, XNORM = DVSC / S.hwhm;
  long ILO = fint(((S.vbot - V1I) / DVSC) + 1.5);
  ILO = std::max(ILO, 1L);
  long IHI = fint(((S.vtop - V1I) / DVSC) + 1.5);
  IHI = std::min<long>(IHI, nc);
  std::vector<double> R1(S.nnhi + 2, 0.);
  for (long I = ILO; I <= IHI; I++) {
    if (sc1[I] == 0.) continue;
    const double ZPEAK = double(I - 1) * RATIO + ZINT;
    long JMAX = fint(ZPEAK + ZBOUND + 1.5);
    long JMIN = fint(ZPEAK - ZBOUND + 1.5);
    JMIN = std::max(JMIN, 1L);
    const double SI = XNORM * sc1[I];
    for (long JF = JMIN; JF <= JMAX && JF <= S.nnhi; JF++) {
      const double ZF = (double(JF - 1) - ZPEAK) * ZSLOPE;
      long IT = fint(std::fabs(ZF) + 1.5);
      if (IT > S.nfmax) IT = S.nfmax;
      R1[JF] = R1[JF] + SI * S.xf[IT];
    }
  }
  out.assign(R1.begin() + 33, R1.begin() + S.nnhi + 1);
  return LBL_OK;
}

}  // namespace

// =========================================================================
// C entry points (called through ctypes by the tests and bench.py)
// =========================================================================
extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

void orc_set_rsym(int on) { g_rsym = on != 0; }


// PATH DV rule (src/lblrtm.f90:5355-5510), standard path (JTYPE=0, IOD=0).
int orc_dv_rule(const lbl_run* R, lbl_layer* Ls, int nlay) {
  double DV = 0.;
  int ISET = R->dvset > 0 ? 1 : 0;
  for (int l = 0; l < nlay; l++) {
    lbl_layer& L = Ls[l];
    double SUMWK = 0.;
    for (int m = 0; m < L.nmol; m++) SUMWK = SUMWK + L.wk[m];
    double WTOTL = SUMWK + L.wbroad;
    double FRH2O = L.wk[0] / WTOTL;
    double ALFCOR = (L.pave / P0) * std::sqrt(TEMP0 / L.tave);
    double H2OSLF = (1. - FRH2O + 5. * FRH2O);
    double ALBAR = R->alfal0 * ALFCOR * H2OSLF;
    double ADBAR = 3.58115E-07 * (0.5 * (R->v1 + R->v2)) * std::sqrt(L.tave / R->avmass);
    double AVBAR = 0.5 * (ALBAR + std::sqrt(ALBAR * ALBAR + 4. * ADBAR * ADBAR));
    double OLDDV = DV;
    DV = AVBAR / R->sample;
    if (DV < R->dvset && ISET == 1) {
      DV = OLDDV;
      if (l == 0 && DV == 0.) DV = R->dvset;
    }
    long ITYPE = 99;
    if (l == 0) {
      long ISCAL = fint(std::log10(DV) - 3.);
      // 10.**ISCAL with an integer exponent: repeated products, reciprocal
      double SCAL = 1.;
      for (long k = 0; k < std::labs(ISCAL); k++) SCAL *= 10.;
      if (ISCAL < 0) SCAL = 1. / SCAL;
      long IDV = fint((DV / SCAL) + 0.5);
      if (IDV % 2 > 0) IDV = IDV + 1;
      DV = SCAL * double(IDV);
    } else {
      double TYPE = OLDDV / DV;
      double TYPMAX = 2.5;
      if (TYPE > TYPMAX) {
        return fail(LBL_E_RANGE, "PATH; ISTOP EQ 1 (DV ratio above 2.5)");
      } else if (TYPE >= 1.2) {
        DV = OLDDV;
        ITYPE = fint(1. / (TYPE - 1.) + 0.5);
        if (ITYPE == 3) ITYPE = 2;
        DV = OLDDV * double(ITYPE) / double(ITYPE + 1);
      } else if (TYPE >= 0.8) {
        DV = OLDDV;
        ITYPE = 0;
      } else {
        DV = OLDDV;
        ITYPE = 0;
        if (R->iemit == 0) {
          ITYPE = fint(TYPE / (1. - TYPE) + 0.5);
          DV = DV * double(ITYPE + 1) / double(ITYPE);
          ITYPE = -ITYPE;
        }
      }
    }
    L.dv = DV;
    L.itype = (int32_t)ITYPE;
  }
  return LBL_OK;
}

int64_t orc_layer_npts(const lbl_run* R, double dv) { return npts_of(*R, dv); }

// SCANFN convolution of a spectrum on v1_in + i*dv_in; *n_out receives the
// output count, out may be NULL to ask for it only.
// SCNINT/INTERP alone: spec (n points from v1_in, spacing dv_in) onto dvo.
int orc_scnint(const double* spec, int64_t n, double v1_in, double dv_in, double dvo, double* out,
               int64_t cap, int64_t* n_out) {
  g_err.clear();
  std::vector<double> res;
  const int rc = orc_scnint_impl(spec, (long)n, v1_in, dv_in, dvo, res);
  if (rc) return rc;
  *n_out = (int64_t)res.size();
  if ((int64_t)res.size() > cap) return fail(LBL_E_ARG, "output capacity");
  for (size_t i = 0; i < res.size(); i++) out[i] = res[i];
  return LBL_OK;
}

int orc_scan(const lbl_scan* sc, const double* spec, int64_t n, double v1_in, double dv_in,
             double* out, int64_t cap, int64_t* n_out, double* dvout) {
  g_err.clear();
  ScanOracle S;
  int rc = scan_setup(*sc, dv_in, S);
  if (rc == LBL_E_RANGE && dv_in > S.dvint && S.dvint > 0.) rc = scan_setup(*sc, S.dvint, S);
  if (rc) return rc;
  *n_out = S.nnhi - 32;
  if (dvout) *dvout = S.dvo;
  if (!out) return LBL_OK;
  std::vector<double> res;
  rc = scan_spectrum(*sc, spec, n, v1_in, dv_in, res);
  if (rc) return rc;
  if ((int64_t)res.size() > cap) return fail(LBL_E_ARG, "output capacity");
  std::copy(res.begin(), res.end(), out);
  return LBL_OK;
}

// PNLINT re-grid of a layer optical depth to DVOUT.  *n_out receives the
// point count; od_out may be NULL to ask for the count only.
int orc_pnlint(const lbl_run* R, double dv, double dvout, const double* od, int64_t n,
               double* od_out, int64_t cap, int64_t* n_out) {
  g_err.clear();
  std::vector<double> res;
  int rc = pnlint_layer(*R, dv, dvout, od, n, &res);
  if (rc) return rc;
  *n_out = (int64_t)res.size();
  if (od_out) {
    if ((int64_t)res.size() > cap) return fail(LBL_E_ARG, "output capacity");
    std::copy(res.begin(), res.end(), od_out);
  }
  return LBL_OK;
}

int orc_layer_od(const lbl_run* R, const lbl_layer* L, const lbl_lines* lines,
                 const lbl_mtckd* ck, int32_t* jrad, double* od, int64_t npts) {
  g_err.clear();
  if (!R || !L || !lines || !jrad || !od) return fail(LBL_E_ARG, "NULL argument");
  Tape3 t3(lines);
  for (int64_t b = 0; b < t3.nb(); b++)
    if (t3.bs[b + 1] - t3.bs[b] > 250) return fail(LBL_E_NREC, "RDLIN; NREC GT LIMIN");
  std::vector<PanelOut> panels;
  int j = *jrad;
  int rc = opdpth(R, L, t3, (R->icntnm ? ck : nullptr), &j, panels);
  if (rc != LBL_OK) return rc;
  int64_t k = 0;
  for (auto& p : panels)
    for (double v : p.r) {
      if (k < npts) od[k] = v;
      k++;
    }
  if (k != npts) return fail(LBL_E_ARG, "npts mismatch: oracle produced " + std::to_string(k));
  *jrad = j;
  return LBL_OK;
}

// One XMERGE step from arrays.  first!=0: ABINIT (iemit 0) / EMINIT.
int orc_merge_layer(const lbl_run* R, const lbl_layer* L, int first,
                    double dv_old, const double* rad_in, const double* tr_in,
                    int64_t n_old, const double* od, double* rad_out,
                    double* tr_out, int64_t n_new) {
  g_err.clear();
  std::vector<PanelOut> kp = panels_from_array(*R, L->dv, od, n_new);
  std::vector<MPanel> out;
  // bit 0: the first layer; bit 1: the last layer (its boundary term, IPATHL=3)
  const bool last = (first & 2) != 0;
  first &= 1;
  if (first) {
    if (R->iemit == 0) {
      for (auto& p : kp) out.push_back(MPanel{p.v1p, p.v2p, p.dvp, p.nlim, p.r, std::vector<double>(p.nlim, 0.)});
    } else {
      eminit(*R, *L, kp, out);
    }
  } else {
    std::vector<PanelOut> op = panels_from_array(*R, dv_old, rad_in, n_old);
    std::vector<MPanel> old;
    std::vector<PanelOut> ot = panels_from_array(*R, dv_old, tr_in ? tr_in : rad_in, n_old);
    for (size_t i = 0; i < op.size(); i++)
      old.push_back(MPanel{op[i].v1p, op[i].v2p, op[i].dvp, op[i].nlim, op[i].r, ot[i].r});
    int rc = (R->iemit == 0) ? absmrg(*L, dv_old, old, kp, out)
                             : radmrg(*R, *L, dv_old, old, kp, out);
    if (rc != LBL_OK) return rc;
  }
  // (a layer that is both first and last goes through EMINIT, which has no
  // boundary term looking up)
  if (last && !first && R->iemit == 1 && R->ipathl == 3) embnd(*R, out);
  int64_t k = 0;
  for (auto& p : out)
    for (long i = 0; i < p.nlim; i++, k++) {
      if (k < n_new) {
        rad_out[k] = p.rad[i];
        if (tr_out) tr_out[k] = p.tr[i];
      }
    }
  return LBL_OK;
}

// Whole standard layer loop for one profile.  layers[].dv/itype computed.
int orc_forward(const lbl_run* R, lbl_layer* Ls, int nlay, const lbl_lines* lines,
                const lbl_mtckd* ck, double* rad, double* tr, int64_t npts) {
  g_err.clear();
  int rc = orc_dv_rule(R, Ls, nlay);
  if (rc != LBL_OK) return rc;
  Tape3 t3(lines);
  int jrad = R->jrad;
  std::vector<MPanel> acc;
  double dv_old = 0.;
  for (int l = 0; l < nlay; l++) {
    std::vector<PanelOut> panels;
    rc = opdpth(R, &Ls[l], t3, (R->icntnm ? ck : nullptr), &jrad, panels);
    if (rc != LBL_OK) return rc;
    std::vector<MPanel> out;
    if (l == 0) {
      if (R->iemit == 0) {
        for (auto& p : panels)
          out.push_back(MPanel{p.v1p, p.v2p, p.dvp, p.nlim, p.r, std::vector<double>(p.nlim, 0.)});
      } else {
        eminit(*R, Ls[l], panels, out);
      }
    } else {
      rc = (R->iemit == 0) ? absmrg(Ls[l], dv_old, acc, panels, out)
                           : radmrg(*R, Ls[l], dv_old, acc, panels, out);
      if (rc != LBL_OK) return rc;
    }
    acc.swap(out);
    dv_old = Ls[l].dv;
  }
  if (R->iemit == 1 && R->ipathl == 3 && nlay > 1) embnd(*R, acc);
  int64_t k = 0;
  for (auto& p : acc)
    for (long i = 0; i < p.nlim; i++, k++)
      if (k < npts) {
        rad[k] = p.rad[i];
        if (tr) tr[k] = p.tr[i];
      }
  if (k != npts) return fail(LBL_E_ARG, "npts mismatch: oracle produced " + std::to_string(k));
  return LBL_OK;
}

// PLANCK_DT (src/xmerge.f90:1019-1080): the factor of the Planck function's
// temperature derivative at XKT, times BBVAL (EMDT passes the layer's
// Planck value for both the layer and the upper level).
double PLANCK_DT_REF(double VI, double XKT, double BBVAL) {
  double v = 0.;
  if (XKT > 0.0) {
    const double VIOKT = VI / XKT, VTKELV = XKT * RADCN2;
    if (VIOKT <= 1e-2) v = 1. / (-VTKELV * (1. + 5e-1 * VIOKT));
    else if (VIOKT <= 80.0) v = VIOKT / (VTKELV * (1. - std::exp(-VIOKT)));
  }
  return v * BBVAL;
}

// dB/dT of the PLANCK function's two branches at temperature t (the
// derivative of the discrete forward model, central-difference mode).
double planck_dt_model(double vi, double t) {
  if (!(t > 0.)) return 0.;
  const double xkt = t / RADCN2;
  const double x = vi / xkt;
  if (x < 1e-2) return RADCN1 * (vi * vi) / RADCN2 * (1. + x) / ((1. + 0.5 * x) * (1. + 0.5 * x));
  if (x > 80.) return 0.;
  const double e = std::exp(-x);
  return RADCN1 * (vi * vi * vi) * e / (1. - e) * (x / t) / (1. - e);
}

// Radiance Jacobians of the upwelling top-of-atmosphere radiance with
// respect to each layer's temperature and the log column amount of the
// listed molecules: the reference's analytic-Jacobian path (lblrtm.f90:
// 2855-3067: one extra OPDPTH per layer and parameter; EMDT xmerge.f90:
// 4406-5030 saves BBEFF, BBSAV, BBASAV, BBDSAV, BBDLSAV, FSAV, dF_dtau;
// TDERIVup :5956-6144 and QDERIVup :5786-5952 form the layer rows), each
// row carried to the top through the later layers' RADNN regrid and
// transmittance (the reference's TRTOTDN product on a common grid).
//   mode 1: the reference's definitions: dtau/dT = tau(T+1 K) - tau where the
//           layer transmittance exceeds 1e-6 (else 0); the molecule row uses
//           the optical depth of a run with that molecule alone (other WK
//           zero, WK(7) added to WBROAD);
//   mode 0: central differences (T +-0.1 K, amount +-1 %) merged with the
//           exact derivative of EMIN/EMINIT/RADNN.
int jacobian(const lbl_run& R, lbl_layer* Ls, int nlay, const lbl_lines* lines,
             const lbl_mtckd* ck, const int* mols, int nq, int mode, double* rad, double* jac,
             int64_t npts) {
  int rc = orc_dv_rule(&R, Ls, nlay);
  if (rc != LBL_OK) return rc;
  if (R.iemit != 1 || R.ipathl != 1) return fail(LBL_E_ARG, "upwelling radiance only");
  Tape3 t3(lines);
  const lbl_mtckd* cku = R.icntnm ? ck : nullptr;
  const int np = 1 + nq;
  std::vector<MPanel> acc;
  std::vector<std::vector<MPanel>> rows((size_t)np * nlay);
  int jrad = R.jrad;
  double dv_old = 0.;
  auto od_of = [&](const lbl_layer& L, int j, std::vector<PanelOut>& out) {
    int jj = j;
    return opdpth(&R, &L, t3, cku, &jj, out);
  };
  for (int l = 0; l < nlay; l++) {
    const lbl_layer& L = Ls[l];
    const int jin = jrad;
    std::vector<PanelOut> od;
    rc = opdpth(&R, &L, t3, cku, &jrad, od);
    if (rc != LBL_OK) return rc;
    // optical-depth inputs of each parameter's row
    std::vector<std::vector<PanelOut>> dp(np);
    for (int k = 0; k < np; k++) {
      if (mode == 0) {
        lbl_layer Lp = L, Lm = L;
        double h;
        if (k == 0) {
          Lp.tave += 0.1;
          Lm.tave -= 0.1;
          h = 0.2;
        } else {
          Lp.wk[mols[k - 1] - 1] *= 1.01;
          Lm.wk[mols[k - 1] - 1] *= 0.99;
          h = std::log(1.01) - std::log(0.99);
        }
        std::vector<PanelOut> pp, pm;
        if ((rc = od_of(Lp, jin, pp)) || (rc = od_of(Lm, jin, pm))) return rc;
        for (size_t q = 0; q < pp.size(); q++)
          for (size_t i = 0; i < pp[q].r.size(); i++) pp[q].r[i] = (pp[q].r[i] - pm[q].r[i]) / h;
        dp[k] = std::move(pp);
      } else {
        lbl_layer Lq = L;
        if (k == 0) {
          Lq.tave = L.tave + 1.;
        } else {
          const int m = mols[k - 1];
          for (int j = 0; j < LBL_WKDIM; j++) Lq.wk[j] = 0.;
          Lq.wk[m - 1] = L.wk[m - 1];
          Lq.wbroad = L.wbroad + L.wk[6];
        }
        if ((rc = od_of(Lq, jin, dp[k]))) return rc;
      }
    }
    // incoming radiance on this layer's grid
    const double XKT = L.tave / RADCN2, XKTA = L.tzu / RADCN2;
    std::vector<MPanel> rin;
    if (l > 0) {
      rc = radmrg_core(R, L, dv_old, acc, od,
                       [&](size_t, const PanelOut& p, std::vector<double>& EM,
                           std::vector<double>& TR) {
                         EM.assign(p.nlim + 1, 0.);
                         TR.assign(p.nlim + 1, 1.);
                       },
                       rin);
      if (rc != LBL_OK) return rc;
    }
    // the layer transmittance and this layer's rows, point by point as EMDT
    std::vector<std::vector<double>> trl(od.size());
    for (int k = 0; k < np; k++) rows[(size_t)k * nlay + l].clear();
    const double TBND = R.tmpbnd, XKTBND = TBND / RADCN2;
    const double rec_6 = 1. / 6.;
    for (size_t q = 0; q < od.size(); q++) {
      const PanelOut& p = od[q];
      trl[q].assign(p.nlim + 1, 0.);
      std::vector<std::vector<double>> d(np, std::vector<double>(p.nlim, 0.));
      double VI = p.v1p;
      for (long I = 1; I <= p.nlim; I++) {
        const double BB = PLANCK(VI, XKT);
        const double bb_dif = XKTA > 0. ? PLANCK(VI, XKTA) - BB : 0.;
        const double tau = p.r[I - 1];
        double odvi = tau;
        const bool clamped = odvi < -OD_LO;
        if (clamped) odvi = -OD_LO;
        const double tr_i = std::exp(-odvi);
        double f_i, df_i;
        if (odvi <= OD_LO) {
          f_i = rec_6 * odvi;
          df_i = rec_6;
        } else {
          f_i = 1. - 2. * (tr_i / (tr_i - 1.) + 1. / odvi);
          df_i = -2. * (tr_i / ((tr_i - 1.) * (tr_i - 1.)) - 1. / (odvi * odvi));
        }
        trl[q][I] = tr_i;
        const double bs = (l == 0 && TBND > 0.) ? PLANCK(VI, XKTBND) * R.bndemi : 0.;
        const double rado = l == 0 ? bs : rin[q].rad[I - 1];
        const double bbeff = BB + bb_dif * f_i;
        for (int k = 0; k < np; k++) {
          const double x = dp[k][q].r[I - 1];
          double v;
          if (mode == 0) {
            const double dem_do = tr_i * bbeff + (1. - tr_i) * bb_dif * df_i;
            const double dr_do = dem_do - tr_i * rado;
            v = clamped ? 0. : dr_do * x;
            if (k == 0)
              v += (1. - tr_i) * (XKTA > 0. ? 1. - f_i : 1.) * planck_dt_model(VI, L.tave);
          } else {
            const double betai = (BB + bb_dif) - BB;
            if (k == 0) {
              const double BBD = PLANCK_DT_REF(VI, XKT, BB);
              const double bbdT = XKTA > 0. ? PLANCK_DT_REF(VI, XKTA, BB) : 0.;
              const double optdpt = tr_i > 1.e-06 ? -std::log(tr_i) : x;
              const double dtaudT = x - optdpt;
              v = (bbeff + betai * f_i - rado) * dtaudT * tr_i + BBD * (1. - tr_i) +
                  (1. - tr_i) * ((bbdT - BBD) * f_i + betai * df_i * dtaudT);
            } else {
              v = x * ((bbeff + betai * f_i - rado) * tr_i + (1. - tr_i) * betai * df_i);
            }
          }
          d[k][I - 1] = v;
        }
        VI = VI + p.dvp;
      }
      for (int k = 0; k < np; k++)
        rows[(size_t)k * nlay + l].push_back(
            MPanel{p.v1p, p.v2p, p.dvp, p.nlim, d[k], std::vector<double>(p.nlim, 0.)});
    }
    // rows of the layers below, carried through this layer
    if (l > 0) {
      for (int k = 0; k < np; k++)
        for (int j = 0; j < l; j++) {
          std::vector<MPanel> out;
          rc = radmrg_core(R, L, dv_old, rows[(size_t)k * nlay + j], od,
                           [&](size_t pi, const PanelOut& p, std::vector<double>& EM,
                               std::vector<double>& TR) {
                             EM.assign(p.nlim + 1, 0.);
                             TR = trl[pi];
                           },
                           out);
          if (rc != LBL_OK) return rc;
          rows[(size_t)k * nlay + j].swap(out);
        }
    }
    // the forward merge
    std::vector<MPanel> out;
    if (l == 0) eminit(R, L, od, out);
    else if ((rc = radmrg(R, L, dv_old, acc, od, out)) != LBL_OK) return rc;
    acc.swap(out);
    dv_old = L.dv;
  }
  int64_t k = 0;
  for (auto& p : acc)
    for (long i = 0; i < p.nlim; i++, k++)
      if (k < npts && rad) rad[k] = p.rad[i];
  if (k != npts) return fail(LBL_E_ARG, "npts mismatch: oracle produced " + std::to_string(k));
  for (int q = 0; q < np; q++)
    for (int l = 0; l < nlay; l++) {
      int64_t i = 0;
      double* dst = jac + ((int64_t)q * nlay + l) * npts;
      for (auto& p : rows[(size_t)q * nlay + l])
        for (long t = 0; t < p.nlim; t++, i++)
          if (i < npts) dst[i] = p.rad[t];
      if (i != npts) return fail(LBL_E_ARG, "Jacobian row length mismatch");
    }
  return LBL_OK;
}

int orc_jacobian(const lbl_run* R, lbl_layer* Ls, int nlay, const lbl_lines* lines,
                 const lbl_mtckd* ck, const int* mols, int nq, int mode, double* rad, double* jac,
                 int64_t npts) {
  g_err.clear();
  if (!R || !Ls || nlay < 1 || !jac || nq < 0 || (nq > 0 && !mols)) return fail(LBL_E_ARG, "bad argument");
  return jacobian(*R, Ls, nlay, lines, ck, mols, nq, mode, rad, jac, npts);
}

// Shape tables for known-answer tests: which = 0..4 -> F1,F2,F3,FG,XVER.
int orc_shape_table(int which, double* out, int n) {
  const Shapes& s = shapes();
  const double* t = which == 0 ? s.F1 : which == 1 ? s.F2 : which == 2 ? s.F3 : which == 3 ? s.FG : s.XVER;
  for (int i = 0; i < n && i < NFMX; i++) out[i] = t[i + 1];
  return LBL_OK;
}

double orc_planck(double v, double t) { return PLANCK(v, t / RADCN2); }
double orc_radfn(double v, double t) { return RADFN(v, t / RADCN2); }
int orc_tips_scor(int mol, int iso, double t, double* scor) {
  double a, b;
  if (!tips_q(mol, iso, 296., &a) || !tips_q(mol, iso, t, &b)) return LBL_E_RANGE;
  *scor = a / b;
  return LBL_OK;
}

// Far-wing diagnostics: number of LBLF4 windows and shrunk lines of a layer.
int orc_far_wing_stats(const lbl_run* R, const lbl_layer* L, const lbl_lines* lines,
                       int64_t* nshrunk, int64_t* nblocks) {
  Tape3 t3(lines);
  Layer S;
  S.R = R;
  S.LY = L;
  S.t3 = &t3;
  S.ck = nullptr;
  S.jrad = 0;
  S.PAVE = L->pave;
  S.TAVE = L->tave;
  S.DV = L->dv;
  S.V1 = R->v1;
  S.V2 = R->v2;
  S.WTOT = L->wbroad;
  for (int m = 0; m < L->nmol; m++) S.WTOT += L->wk[m];
  int rc = molec(*L, S.WTOT, S.mc);
  if (rc) return rc;
  S.DVR4 = 64. * R->sample * S.DV / R->sample;
  S.BOUND4 = 25.;
  S.V1R4 = S.V1 - 2. * S.DVR4;
  S.V2R4 = S.V2 + 2. * S.DVR4;
  linf4(S, S.V1R4 - S.BOUND4 - S.DVR4, S.V2R4 + S.BOUND4 + 2 * S.DVR4);
  int64_t n = 0;
  for (auto& b : S.tape9) n += (int64_t)b.VNU.size();
  *nshrunk = n;
  *nblocks = (int64_t)S.tape9.size();
  return LBL_OK;
}

double orc_brightness_temperature(double v, double rad) {
  return RADCN2 * v / std::log(RADCN1 * v * v * v / rad + 1.);
}

}  // extern "C"
