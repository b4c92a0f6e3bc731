// lbl_plan.cpp -- host-side planning: DV rule, per-layer constants, panel
// and far-wing window schedule, line-index ranges.  Compiled without FMA
// contraction so the FP64 schedule arithmetic rounds exactly as the
// reference's does (each product and sum rounded separately).
#include "lbl_plan.h"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "../data/ref_tables.h"

namespace lbl {
namespace {

const double PI = 3.1415926535898;        // src/phys_consts.f90:66
const double BOLTZ = 1.3806503E-16;
const double CLIGHT = 2.99792458E+10;
const double AVOGAD = 6.02214199E+23;
const double RADCN2 = 1.4387752;
const double ONEPL = 1.001;
const double P0 = 1013.25, TEMP0 = 296.;   // src/lblrtm.f90:2115-2116
const double HWF3 = 64.;
const double DXF1 = 0.002, DXF2 = 0.008, DXF3 = 0.032;
const double TEMPLC[5] = {0., 200., 250., 296., 340.};

inline long fint(double x) { return (long)x; }

// Radiation term (RADFN, src/oprop.f90:2235-2296).
double radfn(double vi, double xkt) {
  if (xkt > 0.0) {
    double x = vi / xkt;
    if (x <= 0.01) return 0.5 * x * vi;
    if (x <= 10.0) {
      double e = std::exp(-x);
      return vi * (1. - e) / (1. + e);
    }
  }
  return vi;
}

// Lagrange 3/4-point table recall of TIPS (AtoB, src/oprop.f90:11708).
double lagrange_recall(double t, const double* T, const double* Q, int n) {
  auto nz = [](double d) { return d == 0. ? 0.0001 : d; };
  for (int i = 1; i < n; i++) {            // 0-based i <-> Fortran I = i+1
    if (T[i] < t) continue;
    int I = i + 1;
    if (I < 3 || I == n) {
      int J = (I < 3) ? 3 : n;
      const double a0 = T[J - 3], a1 = T[J - 2], a2 = T[J - 1];
      double w0 = (t - a1) * (t - a2) / (nz(a0 - a1) * nz(a0 - a2));
      double w1 = (t - a0) * (t - a2) / (nz(a1 - a0) * nz(a1 - a2));
      double w2 = (t - a0) * (t - a1) / (nz(a2 - a0) * nz(a2 - a1));
      return w0 * Q[J - 3] + w1 * Q[J - 2] + w2 * Q[J - 1];
    }
    const double a0 = T[I - 3], a1 = T[I - 2], a2 = T[I - 1], a3 = T[I];
    double w0 = (t - a1) * (t - a2) * (t - a3);
    w0 = w0 / (nz(a0 - a1) * nz(a0 - a2) * nz(a0 - a3));
    double w1 = (t - a0) * (t - a2) * (t - a3);
    w1 = w1 / (nz(a1 - a0) * nz(a1 - a2) * nz(a1 - a3));
    double w2 = (t - a0) * (t - a1) * (t - a3);
    w2 = w2 / (nz(a2 - a0) * nz(a2 - a1) * nz(a2 - a3));
    double w3 = (t - a0) * (t - a1) * (t - a2);
    w3 = w3 / (nz(a3 - a0) * nz(a3 - a1) * nz(a3 - a2));
    return w0 * Q[I - 3] + w1 * Q[I - 2] + w2 * Q[I - 1] + w3 * Q[I];
  }
  return 0.;
}

bool partition_q(int mol, int iso, double t, double* q) {
  if (mol < 1 || mol > LBL_NQMOL || iso < 1 || iso > LBL_QNISO[mol - 1]) return false;
  if (t < 70. || t > 3000.) return false;
  *q = lagrange_recall(t, LBL_TDAT, LBL_QOFT[mol - 1][iso - 1], 119);
  return true;
}

}  // namespace

void build_shape_tables(ShapeTables* t) {
  // Sub-functions of the approximate Voigt shape (SHAPEL/SHAPEG/VERFN,
  // src/oprop.f90:1822-1991): F1 = L - Q1 on 0..4, F2 = Q1 - Q2 (then
  // L - Q2) on 0..16, F3 = Q2 - Q3 (then L - Q3) on 0..64, with
  // Q_k(x^2) = A(z_k) + B(z_k) x^2 matching the Lorentzian L at z_k.
  std::memset(t, 0, sizeof(*t));
  const double rpi = 1. / (2. * std::asin(1.));
  auto A = [](double z) { return (1. + 2. * z * z) / std::pow(1. + z * z, 2); };
  auto B = [](double z) { return -1. / std::pow(1. + z * z, 2); };
  const double a1 = A(4.), b1 = B(4.), a2 = A(16.), b2 = B(16.), a3 = A(64.), b3 = B(64.);
  auto lor = [](double x2) { return 1. / (1. + x2); };
  t->f1[1] = rpi * (lor(0.) - a1);
  for (int j = 2; j <= 2001; j++) {
    double x = double(j - 1) * DXF1, x2 = x * x;
    t->f1[j] = rpi * (lor(x2) - (a1 + b1 * x2));
  }
  t->f1[2001] = 0.;
  t->f2[1] = rpi * (a1 - a2);
  long j1 = fint(4. / DXF2 + 1.001);
  for (long j = 2; j <= 2001; j++) {
    double x = double(j - 1) * DXF2, x2 = x * x;
    t->f2[j] = (j <= j1) ? rpi * ((a1 + b1 * x2) - (a2 + b2 * x2))
                         : rpi * (lor(x2) - (a2 + b2 * x2));
  }
  t->f2[2001] = 0.;
  t->f3[1] = rpi * (a2 - a3);
  long j2 = fint(16. / DXF3 + 1.001);
  for (long j = 2; j <= 2001; j++) {
    double x = double(j - 1) * DXF3, x2 = x * x;
    t->f3[j] = (j <= j2) ? rpi * ((a2 + b2 * x2) - (a3 + b3 * x2))
                         : rpi * (lor(x2) - (a3 + b3 * x2));
  }
  const double ln2 = std::log(2.);
  const double gnorm = std::sqrt(ln2 * rpi);
  t->fg[1] = gnorm * std::exp(-ln2 * 0.);
  for (int j = 2; j <= 2001; j++) {
    double x = double(j - 1) * DXF1;
    t->fg[j] = gnorm * std::exp(-ln2 * (x * x));
  }
  t->fg[2001] = 0.;
  const double cexp = 0.45, ce0 = 1., ce2 = -.20737285249, ce4 = -.00872684335747;
  const double se0 = std::sqrt(cexp / PI), ae2 = 2. * cexp, ae4 = ae2 * ae2 / 3.;
  for (int i = 1; i <= kNfmx; i++) {
    double z = DXF1 * double(i - 1), z2 = z * z;
    double xe0 = se0 * std::exp(-cexp * z2);
    t->xver[i] = (1. / (ce0 + ce2 + ce4)) * (ce0 + ce2 * ae2 * z2 + ce4 * ae4 * z2 * z2) * xe0;
  }
}

int dv_rule(const lbl_run& R, lbl_layer* Ls, int nlay, std::string* err) {
  double dv = 0.;
  const bool iset = R.dvset > 0.;
  for (int l = 0; l < nlay; l++) {
    lbl_layer& L = Ls[l];
    if (L.nmol < 1 || L.nmol > LBL_WKDIM || L.pave <= 0. || L.tave <= 0.) {
      *err = "layer " + std::to_string(l) + ": bad nmol/pave/tave";
      return LBL_E_ARG;
    }
    if (R.iemit == 1 && (R.ipathl == 2 || (R.ipathl == 1 && R.bndrfl > 0.)) && !(L.tzl > 0.)) {
      // the tangent path's far crossing and the reflected atmosphere's
      // downward emission radiate at TZL (XKTB)
      *err = "layer " + std::to_string(l) +
             ": the tangent path and the reflected atmosphere need TZL > 0";
      return LBL_E_ARG;
    }
    double sumwk = 0.;
    for (int m = 0; m < L.nmol; m++) sumwk = sumwk + L.wk[m];
    double wtotl = sumwk + L.wbroad;
    double frh2o = L.wk[0] / wtotl;
    double alfcor = (L.pave / P0) * std::sqrt(TEMP0 / L.tave);
    double h2oslf = (1. - frh2o + 5. * frh2o);
    double albar = R.alfal0 * alfcor * h2oslf;
    double adbar = 3.58115E-07 * (0.5 * (R.v1 + R.v2)) * std::sqrt(L.tave / R.avmass);
    double avbar = 0.5 * (albar + std::sqrt(albar * albar + 4. * adbar * adbar));
    double olddv = dv;
    dv = avbar / R.sample;
    if (dv < R.dvset && iset) {
      dv = olddv;
      if (l == 0 && dv == 0.) dv = R.dvset;
    }
    long itype = 99;
    if (l == 0) {
      long iscal = fint(std::log10(dv) - 3.);
      double scal = 1.;
      for (long k = 0; k < std::labs(iscal); k++) scal *= 10.;
      if (iscal < 0) scal = 1. / scal;
      long idv = fint((dv / scal) + 0.5);
      if (idv % 2 > 0) idv = idv + 1;
      dv = scal * double(idv);
    } else {
      double type = olddv / dv;
      if (type > 2.5) {
        *err = "DV rule: OLDDV/DV above 2.5 at layer " + std::to_string(l) +
               " ('PATH; ISTOP EQ 1')";
        return LBL_E_RANGE;
      } else if (type >= 1.2) {
        itype = fint(1. / (type - 1.) + 0.5);
        if (itype == 3) itype = 2;
        dv = olddv * double(itype) / double(itype + 1);
      } else if (type >= 0.8) {
        dv = olddv;
        itype = 0;
      } else {
        dv = olddv;
        itype = 0;
        if (R.iemit == 0) {
          itype = fint(type / (1. - type) + 0.5);
          dv = dv * double(itype + 1) / double(itype);
          itype = -itype;
        }
      }
    }
    L.dv = dv;
    L.itype = (int32_t)itype;
  }
  return LBL_OK;
}

int64_t layer_npts(const lbl_run& R, double dv) {
  double vft = R.v1 - 32. * dv;
  int64_t n = 0;
  for (;;) {
    long nhi = 2432;
    if ((vft + double(nhi - 1) * dv) > R.v2) {
      nhi = fint((R.v2 - vft) / dv + 1.);
      double v2p = vft + double(nhi - 1) * dv;
      if (v2p < R.v2) nhi = nhi + 1;
      return n + (nhi - 33 + 1);
    }
    n += 2400;
    vft = vft + double(kNlim1 - 1) * dv;
  }
}

int next_jrad(const lbl_run& R, const lbl_layer& L, int jrad) {
  double xkt = L.tave / RADCN2;
  if (((R.v1 / xkt) < 5.) && (jrad != -1)) return 0;
  return jrad;
}

int plan_layer(const lbl_run& R, const lbl_layer& L, int jrad_in, const HostLines& H,
               LayerPlan* P, std::string* err) {
  const double* vnu = H.vnu;
  const int64_t nlines = H.n;
  const int64_t* bs = H.bs;
  const int64_t nblk = H.nblk;
  LayerDev& d = P->d;
  std::memset(&d, 0, sizeof(d));
  if (L.nmol < 1 || L.nmol > kNMolTab) {
    *err = "nmol must be 1..7 (molecules with TIPS tables)";
    return LBL_E_RANGE;
  }
  if (!(L.dv > 0.)) {
    *err = "layer dv not set (run lbl_dv_rule)";
    return LBL_E_ARG;
  }
  if (L.tave < 70. || L.tave > 3000.) {
    *err = "layer temperature outside the TIPS range 70-3000 K";
    return LBL_E_RANGE;
  }
  const double DV = L.dv;
  d.pave = L.pave;
  d.tave = L.tave;
  d.dv = DV;
  d.v1 = R.v1;
  d.v2 = R.v2;
  d.nmol = L.nmol;
  d.jrad = next_jrad(R, L, jrad_in);
  d.ilblf4 = R.ilblf4;
  d.icntnm = R.icntnm;
  d.xkt = L.tave / RADCN2;
  const double xkt0 = TEMP0 / RADCN2;
  d.betacr_n = (1. / d.xkt) - (1. / xkt0);
  d.beta_f = RADCN2 / L.tave;
  d.betacr_f = d.beta_f - RADCN2 / TEMP0;
  d.tratio = L.tave / TEMP0;
  d.rhorat = (L.pave / P0) * (TEMP0 / L.tave);
  d.pavp0 = L.pave / P0;
  d.pavp2 = d.pavp0 * d.pavp0;
  // line-coupling temperature brackets: LNCOR1 (:989-997) and LINF4 (:3124-3130)
  long ilc = 1;
  for (long il = 1; il <= 3; il++) {
    ilc = il;
    if (L.tave < TEMPLC[ilc + 1]) break;
  }
  d.ilc_n = (int32_t)ilc;
  d.rectlc_n = 1.0 / (TEMPLC[ilc + 1] - TEMPLC[ilc]);
  d.tmpdif_n = L.tave - TEMPLC[ilc];
  for (ilc = 1; ilc <= 4; ilc++)
    if (L.tave <= TEMPLC[ilc]) break;
  if (ilc == 1) ilc = 2;
  if (ilc == 5) ilc = 4;
  d.ilc_f = (int32_t)ilc;
  d.rectlc_f = 1.0 / (TEMPLC[ilc] - TEMPLC[ilc - 1]);
  d.tmpdif_f = L.tave - TEMPLC[ilc];

  // MOLEC IND=2 (src/oprop.f90:2535-2552) with TIPS_2003 scor = Q(296)/Q(T)
  double wtot = L.wbroad;
  for (int m = 0; m < L.nmol; m++) wtot += L.wk[m];
  d.h2o_fac = L.wk[0] / wtot;
  d.wtot = wtot;
  const double fad = std::log(2.) * 2. * AVOGAD * BOLTZ / (CLIGHT * CLIGHT);
  for (int m = 1; m <= L.nmol; m++) {
    d.wk[m] = L.wk[m - 1];
    d.rhoslf[m] = d.rhorat * L.wk[m - 1] / wtot;
    d.isomax[m] = LBL_ISO_MAX[m - 1];
    for (int iso = 1; iso <= LBL_ISO_MAX[m - 1]; iso++) {
      double q296, qt;
      if (!partition_q(m, iso, 296., &q296) || !partition_q(m, iso, L.tave, &qt)) {
        *err = "TIPS table missing";
        return LBL_E_RANGE;
      }
      d.scor[m][iso] = q296 / qt;
      d.alfd1[m][iso] = std::sqrt(fad * L.tave / LBL_SMASS[m - 1][iso - 1]);
    }
  }

  // HIRAC1 constants (src/oprop.f90:229-307)
  d.dptmn = R.dptmin;
  if (d.jrad != 1) d.dptmn = R.dptmin / radfn(R.v2, L.tave / RADCN2);
  d.dptfc = R.dptfac;
  d.alfmax = 4 * R.sample * DV * 0.04 / R.alfal0;
  long nalfmax = fint(d.alfmax / DV);
  long nbound = fint((2. * HWF3) * double(nalfmax) + 0.01);
  long max1 = kNShift + kNlim1 + kNShift + nbound / 2;
  max1 = max1 + 4 * nalfmax;
  d.max1 = max1;
  d.bound = double(nbound) * DV / 2.;
  d.dvr2 = (DXF2 / DXF1) * DV;
  d.dvr3 = (DXF3 / DXF1) * DV;
  d.conf2 = DV / d.dvr2;
  d.conf3 = DV / d.dvr3;
  d.wavdxf = DV / DXF1;
  d.vft0 = R.v1 - double(kNShift) * DV;
  d.vbot = R.v1 - d.bound;
  d.vtop = R.v2 + d.bound;

  // continuum grid (OPDPTH, src/lblrtm.f90:6216-6228)
  if (R.icntnm != 0) {
    d.dvabs = 1.;
    d.v1abs = (double)fint(R.v1);
    if (R.v1 < 0.) d.v1abs = d.v1abs - 1.;
    d.v1abs = d.v1abs - 3. * d.dvabs;
    d.v2abs = (double)fint(R.v2 + 3. * d.dvabs + 0.5);
    d.nptabs = fint((d.v2abs - d.v1abs) / d.dvabs + 1.5);
  }

  // far-wing grid (OPDPTH, src/lblrtm.f90:6232-6256)
  double v1r4st = 0., v2r4st = 0.;
  if (R.ilblf4 >= 1) {
    double alfav = R.sample * DV;
    double alfav4 = 64. * alfav;
    d.dvr4 = alfav4 / R.sample;
    d.bound4 = 25.;
    if (R.ilblf4 == 2 && L.pave <= 0.5) d.bound4 = 5.;
    v1r4st = R.v1 - 2. * d.dvr4;
    v2r4st = R.v2 + 2. * d.dvr4;
    d.v1l4 = v1r4st - d.bound4 - d.dvr4;
    d.v2l4 = v2r4st + d.bound4 + 2 * d.dvr4;
  }
  const double dptmn4 = R.dptmin / radfn(v2r4st, L.tave / RADCN2);
  P->win.clear();
  auto add_window = [&](double v1w, int first_panel) {
    WinDev w;
    w.v1r4 = v1w;
    long npt = fint((v2r4st - v1w) / d.dvr4 + ONEPL);
    npt = std::min<long>(npt, kLimOut);
    w.nptr4 = (int32_t)npt;
    w.v2r4 = v1w + d.dvr4 * double(npt - 1);
    w.vlo = w.v1r4 - d.bound4;
    w.vhi = w.v2r4 + d.bound4;
    w.vnulst = w.v2r4 + d.bound4;
    w.dptmn = dptmn4;
    w.first_panel = first_panel;
    P->win.push_back(w);
  };
  if (R.ilblf4 >= 1) add_window(v1r4st, 0);

  // panel loop: accumulated VFT_p, last-panel rule, window refreshes
  P->vft.clear();
  P->win_of.clear();
  double vft = d.vft0;
  const long n2r3 = 155;
  long nhi_last = 0;
  for (long p = 0;; p++) {
    P->vft.push_back(vft);
    P->win_of.push_back((int32_t)P->win.size() - 1);
    long nhi = 2432;
    bool stop = false;
    if ((vft + double(nhi - 1) * DV) > R.v2) {
      nhi = fint((R.v2 - vft) / DV + 1.);
      double v2p = vft + double(nhi - 1) * DV;
      if (v2p < R.v2) nhi = nhi + 1;
      stop = true;
    }
    vft = vft + double(kNlim1 - 1) * DV;
    if (stop) {
      nhi_last = nhi;
      break;
    }
    if (R.ilblf4 >= 1) {
      const WinDev& cur = P->win.back();
      double vf1 = vft - 2. * d.dvr4;
      vf1 = R.v1 + std::floor((vf1 - R.v1) / d.dvr4) * d.dvr4;
      double vf2 = vft + 2. * d.dvr4 + double(n2r3 + 4) * d.dvr3;
      if (vf2 > cur.v2r4 && cur.v2r4 != v2r4st) add_window(vf1, (int)p + 1);
    }
  }
  d.npanel = (int64_t)P->vft.size();
  d.npts = 2400 * (d.npanel - 1) + (nhi_last - 33 + 1);
  d.nwin = (int32_t)P->win.size();
  if (d.npts != layer_npts(R, DV)) {
    *err = "internal: panel count mismatch";
    return LBL_E_ARG;
  }
  // global grid extents: R1 index g1 covers output points 33..32+npts plus
  // the interpolation stencil; R2/R3 their 4- and 16-fold coarser images.
  d.n_r1 = 32 + d.npts + 8;
  d.n_r2 = d.n_r1 / 4 + 8;
  d.n_r3 = d.n_r2 / 4 + 8;

  // ---- line-index ranges ------------------------------------------------
  auto lower = [&](double v) { return int64_t(std::lower_bound(vnu, vnu + nlines, v) - vnu); };
  auto block_of = [&](int64_t i) {
    return int64_t(std::upper_bound(bs, bs + nblk + 1, i) - bs) - 1;
  };
  // RDLIN (src/oprop.f90:741-875): panels with VMAX < VBOT are skipped; in
  // the first panel read, lines below VBOT are skipped; in each panel the
  // range ends at the first record (IFLG>=0, MOL>0) beyond VTOP, and when
  // that record is the panel's last one the next panel is read as well.
  d.near_lo = d.near_hi = 0;
  d.blk_lo = d.blk_hi = 0;
  {
    int64_t b = 0;
    while (b < nblk && vnu[bs[b + 1] - 1] < d.vbot) b++;
    if (b < nblk) {
      int64_t lo = bs[b];
      if (vnu[bs[b]] < d.vbot) {
        int64_t last_ok = -1;
        lo = -1;
        for (int64_t i = bs[b]; i < bs[b + 1]; i++) {
          if (H.iflg[i] < 0) continue;
          last_ok = i;
          if (vnu[i] >= d.vbot) { lo = i; break; }
        }
        if (lo < 0) lo = last_ok >= 0 ? last_ok : bs[b];
      }
      d.near_lo = lo;
      d.blk_lo = b;
      int64_t hi = nlines;  // EOF unless a stop is found
      // panels whose last line is <= VTOP hold no stop record: jump to the
      // first panel reaching beyond VTOP
      int64_t bb = b;
      {
        const int64_t first_above = int64_t(std::upper_bound(vnu, vnu + nlines, d.vtop) - vnu);
        if (first_above < nlines) bb = std::max(b, block_of(first_above));
        else bb = nblk;
      }
      int64_t from = (bb == b) ? lo : (bb < nblk ? bs[bb] : nlines);
      while (bb < nblk) {
        int64_t last_ok = -1, stop_at = -1;
        for (int64_t i = from; i < bs[bb + 1]; i++) {
          if (H.iflg[i] < 0) continue;
          last_ok = i;
          if (stop_at < 0 && H.mol[i] > 0 && vnu[i] > d.vtop) stop_at = i;
        }
        if (stop_at >= 0 && stop_at != last_ok) { hi = stop_at + 1; break; }
        bb++;
        if (bb < nblk) from = bs[bb];
        if (stop_at >= 0 && bb >= nblk) { hi = stop_at + 1; break; }
      }
      d.near_hi = std::max(hi, lo);
      d.blk_hi = d.near_hi > d.near_lo ? block_of(d.near_hi - 1) + 1 : d.blk_lo;
    } else {
      d.near_lo = d.near_hi = nlines;
      d.blk_lo = d.blk_hi = nblk;
    }
  }
  // LINF4 (src/oprop.f90:3136-3220): lines with VNU >= V1L4 whose strength
  // times amount is non-zero, up to and including the first such line whose
  // pressure-shifted centre lies beyond V2L4.
  if (R.ilblf4 >= 1) {
    d.far_lo = lower(d.v1l4);
    int64_t hi = nlines;
    // a line can pass VHI only if its unshifted centre is within the largest
    // pressure shift of it: start the search there
    const double reach = std::fabs(d.rhorat) * H.max_abs_pshift;
    const int64_t start = std::max(d.far_lo, lower(d.v2l4 - reach - 1e-9));
    for (int64_t i = start; i < nlines; i++) {
      if (H.iflg[i] < 0) continue;
      int m = H.mol[i] % 100, iso = (H.mol[i] % 1000) / 100;
      if (m < 1 || m > LBL_MXMOL || iso < 1 || iso > LBL_ISO_MAX[m - 1]) continue;
      double wkm = (m <= L.nmol) ? L.wk[m - 1] : 0.;
      if ((double)H.sp[i] * wkm == 0.) continue;
      if (vnu[i] < d.v1l4) continue;
      if (vnu[i] + d.rhorat * (double)H.pshift[i] > d.v2l4) { hi = i + 1; break; }
    }
    d.far_hi = hi;
    d.fblk_lo = d.far_lo < nlines ? block_of(d.far_lo) : nblk;
    d.fblk_hi = d.far_hi > d.far_lo ? block_of(d.far_hi - 1) + 1 : d.fblk_lo;
  } else {
    d.far_lo = d.far_hi = 0;
    d.fblk_lo = d.fblk_hi = 0;
  }
  return LBL_OK;
}

// PNLINT's panel loop (src/oprop.f90:1620-1800) replayed per PANEL output
// panel (src/oprop.f90:1435-1451: V1P = VFT+(NLO-1)*DV, V2P by the
// last-panel rule, VFT advanced by NLIM1-1 = 2400 points).  Segments are
// recorded in place of the interpolation loop (label 30); every test,
// truncation and accumulation follows the reference's order.
int pnlint_plan(const lbl_run& R, double dv, double dvout, PnlPlan* P, std::string* err) {
  P->seg.clear();
  P->n_out = 0;
  if (!(dv > 0.) || !(dvout > 0.)) {
    *err = "DV and DVOUT must be positive";
    return LBL_E_ARG;
  }
  for (int jp = 0; jp <= 100; jp++) {
    double apg = jp, p = 0.01 * apg;
    P->a[0][jp] = -p * (p - 1.0) * (p - 2.0) / 6.0;
    P->a[1][jp] = (p * p - 1.0) * (p - 2.0) * 0.5;
    P->a[2][jp] = -p * (p + 1.0) * (p - 2.0) * 0.5;
    P->a[3][jp] = p * (p * p - 1.0) / 6.0;
  }
  P->copy = (dv == dvout) || std::fabs(dvout - dv) < 1.e-8;
  if (P->copy) {
    P->n_out = layer_npts(R, dv);
    return LBL_OK;
  }
  if (dvout > dv) {
    *err = "DVOUT MUST BE < DV";
    return LBL_E_ARG;
  }
  const int limout = 2400;
  double vft = R.v1 - double(kNShift) * dv;
  double v1po = 0.;
  long nlim1 = 1;
  int64_t kq = 0;  // global output index of the open output panel's II=1
  for (int64_t p = 0;; p++) {
    long nhi = 2432;
    double v2p;
    bool istop = false;
    if ((vft + double(nhi - 1) * dv) > R.v2) {
      nhi = fint((R.v2 - vft) / dv + 1.);
      v2p = vft + double(nhi - 1) * dv;
      if (v2p < R.v2) {
        v2p = v2p + dv;
        nhi = nhi + 1;
      }
      istop = true;
    } else {
      v2p = vft + double(nhi - 1) * dv;
    }
    const long nlim = nhi - (kNShift + 1) + 1;
    const double v1p = vft + double(kNShift) * dv;
    // ---- PNLINT entry
    int nppanl = 1;
    int flags = istop ? 2 : 0;
    if (v1po == 0.0) {
      v1po = v1p;
      nlim1 = 1;
      flags |= 1;
    }
    if (istop) v2p = v2p + 2. * dv;
    bool ilast = false;
    for (;;) {
      double v2po = v1po + double(limout) * dvout;
      if (v2p <= v2po + dv && !ilast && nppanl <= 0) break;
      long nlim2;
      if ((v1po + double(limout - 1) * dvout) > R.v2) {
        nlim2 = fint((R.v2 - v1po) / dvout + 1.);
        v2po = v1po + double(nlim2 - 1) * dvout;
        if (v2po < R.v2) {
          v2po = v2po + dvout;
          nlim2 = nlim2 + 1;
        }
        ilast = true;
        if (!istop && v2po > v2p - dv) {
          nlim2 = fint(((v2p - dv - v1po) / dvout) + 1.);
          v2po = v1po + double(nlim2 - 1) * dvout;
          if (v2po + dvout < v2p - dv) {
            nlim2 = nlim2 + 1;
            v2po = v2po + dvout;
          }
          ilast = false;
        }
      } else {
        nlim2 = limout;
        v2po = v1po + double(nlim2 - 1) * dvout;
        if (v2po > v2p - dv) {
          nlim2 = fint(((v2p - dv - v1po) / dvout) + 1.);
          v2po = v1po + double(nlim2 - 1) * dvout;
          if (v2po + dvout < v2p - dv) {
            nlim2 = nlim2 + 1;
            v2po = v2po + dvout;
          }
        }
        ilast = false;
      }
      if (nlim2 >= nlim1 && nlim1 >= 1) {
        PnlSeg s;
        s.v1po = v1po;
        s.v1p = v1p;
        s.fj1dif = (v1po - v1p) / dv + 1. + 2.;
        s.k0 = kq;
        s.g0 = 2400 * p;
        s.ii_lo = (int32_t)nlim1;
        s.ii_hi = (int32_t)nlim2;
        s.nlim = (int32_t)nlim;
        s.flags = flags;
        P->seg.push_back(s);
      }
      if (nlim2 == limout || ilast) {
        kq += nlim2;
        nlim1 = 1;
        nppanl = 0;
        v1po = v2po + dvout;
        if ((v1po + double(limout) * dvout) > (v2p - dv)) nppanl = 1;
      } else {
        nlim1 = nlim2 + 1;
        nppanl = -1;
      }
      if (ilast) break;
    }
    if (ilast) {
      P->n_out = kq;
      return LBL_OK;
    }
    vft = vft + double(kNlim1 - 1) * dv;
    if (istop) {
      *err = "internal: PNLINT did not reach V2";
      return LBL_E_ARG;
    }
  }
}

// SCANFN's set-up (src/postsub.f90:25-420): the function's extent, table
// step and sampling (HWJ, DXJ, NJ, NJMX, SMPLJ, XSCAL :97-117), SAMPL, the
// output spacing DVO = HWHM/SAMPLE and the bound, PANLSC's last point
// (:1600-1660), the shapes (SHAPET :1377-1400, SHAPEG src/oprop.f90:
// 1912-1942, SINCSQ :2445-2484, SINC :2486-2525), SHRKSC's ratio
// (:1276-1320) and CONVSC's constants (:1516-1560).
int scan_plan(const lbl_scan& sc, double dv_in, ScanPlan* P, std::string* err) {
  static const double HWJ[7] = {1., 2., 4., 54.1826, 119.332818, 1., 1.};
  static const double DXJ[7] = {0., 0.02, 0.02, 0.02, 0.02, 0., 0.};
  static const int64_t NJ[7] = {0, 101, 201, 2710, 5968, 0, 0};
  static const int64_t NJMX[7] = {0, 251, 251, 2760, 6018, 0, 0};
  static const double SMPLJ[7] = {.5, 2., 4., 4., 4., .5, .5};
  static const double XSCAL[7] = {0., 0., 0., 1.391557377, 1.89549425, 0., 0.};
  static const long JRATIO[25] = {0, 1, 2, 3, 4, 5, 6, 8, 10, 12, 15, 16, 20,
                                  24, 25, 30, 32, 40, 48, 50, 60, 75, 80, 100, 120};
  const double pi = 2. * std::asin(1.);
  double hwhm = sc.hwhm;
  int jfn = sc.jfn;
  if (!(hwhm > 0.) || !(sc.v2 > sc.v1) || !(dv_in > 0.)) {
    *err = "scan: HWHM, V1 < V2 and the input spacing must be positive";
    return LBL_E_ARG;
  }
  if (jfn < 0) {
    jfn = -jfn;
    if (jfn != 3 && jfn != 4) {
      *err = "SCANFN; INVALID JFN";
      return LBL_E_ARG;
    }
  }
  if (jfn < 0 || jfn > 6) {
    *err = "scan: JFN must be 0-6 (rectangle, triangle, Gaussian, sinc^2, sinc, field-of-view "
           "boxes centred / left-aligned)";
    return LBL_E_ARG;
  }
  const double xscale = XSCAL[jfn];
  if (sc.jfn < 0) hwhm = hwhm / (pi / xscale);
  P->jfn = jfn;
  P->hwf = HWJ[jfn];
  P->dxf = DXJ[jfn];
  P->nf = NJ[jfn];
  P->nfmax = NJMX[jfn];
  double sample = SMPLJ[jfn];
  if (sc.sampl < 0.) sample = hwhm / (-sc.sampl);
  else if (sc.sampl > 0.) sample = sc.sampl;
  // DVINT (SCANFN :245-265): for JFN 5/6 a twelfth of the first box, whose
  // width is V1 BFOV^2 / 2
  const double dvint = (jfn == 5 || jfn == 6)
                           ? sc.v1 * ((hwhm * 3.141592654 / 180.) * (hwhm * 3.141592654 / 180.)) / 24
                           : hwhm / 12.;
  P->dvint = dvint;
  if (dv_in > dvint) {
    *err = "scan: input spacing above DVINT (interpolate first, SCNINT)";
    return LBL_E_RANGE;
  }
  P->hwhm = hwhm;
  P->dvo = hwhm / sample;
  if (jfn == 5 || jfn == 6) {
    // boxes whose width grows with wavenumber (CNVVRC :1986-2214 centred at
    // V1 + (NB-1) DVO, CNVVRL :2216-2440 starting there), up to V2
    P->bfov = hwhm * 3.141592654 / 180.;
    int64_t nb = 1;
    while (sc.v1 + double(nb) * P->dvo <= sc.v2) nb++;
    P->n_out = nb;
    P->nnhi = nb + kNShift;
    return LBL_OK;
  }
  if (jfn == 0) {
    // adjacent boxes of 2 HWHM (SCANFN :393-399, CNVRCT :1779-1985): DVO a
    // whole number IRATIO of input steps; the boxes centred at V1 + (NB-1)
    // DVO up to V2
    const long iratio = fint(P->dvo / dv_in + 0.5);
    P->dvo = double(iratio) * dv_in;
    if (iratio < 2) {
      *err = "scan: IRATIO LESS THAN 2, NO SCANFN";
      return LBL_E_RANGE;
    }
    int64_t nb = 1;
    while (sc.v1 + double(nb) * P->dvo <= sc.v2) nb++;
    P->n_out = nb;
    P->nnhi = nb + kNShift;
    return LBL_OK;
  }
  const long nbound = fint((2. * P->hwf) * sample + 0.01);
  P->bound = double(nbound) * P->dvo / 2.;
  P->vft0 = sc.v1 - double(kNShift) * P->dvo;
  P->vbot = sc.v1 - P->bound;
  P->vtop = sc.v2 + P->bound;
  P->nnhi = fint((sc.v2 - P->vft0) / P->dvo + 1.5);
  P->n_out = P->nnhi - kNShift;
  if (P->n_out < 1 || P->n_out > (int64_t(1) << 30)) {
    *err = "scan: output grid size";
    return LBL_E_RANGE;
  }
  P->xf.assign(P->nfmax + 2, 0.);
  double* xf = P->xf.data();
  if (jfn == 1) {
    xf[1] = 0.5;
    for (int64_t i = 2; i <= P->nf; i++) xf[i] = 0.5 * (1. - 0.5 * (double(i - 1) * P->dxf));
  } else if (jfn == 2) {
    const double fln2 = std::log(2.), recpi = 1. / (2. * std::asin(1.));
    const double fgnorm = std::sqrt(fln2 * recpi);
    xf[1] = fgnorm * std::exp(-fln2 * 0.);
    for (int64_t j = 2; j <= P->nf; j++) {
      const double x = double(j - 1) * P->dxf;
      xf[j] = fgnorm * std::exp(-fln2 * (x * x));
    }
    xf[P->nf] = 0.;
  } else {
    const double xnorm = xscale / pi;
    xf[1] = xnorm;
    for (int64_t i = 2; i <= P->nf; i++) {
      const double a = (double(i - 1) * P->dxf) * xscale;
      const double sx = std::sin(a) / a;
      xf[i] = (jfn == 3) ? xnorm * (sx * sx) : xnorm * sx;
    }
  }
  // SHRKSC
  double dvsc = hwhm / 12.;
  long ir = fint(dvsc / dv_in + 0.5);
  for (int i = 2; i <= 24; i++)
    if (JRATIO[i] > ir) {
      ir = JRATIO[i - 1];
      break;
    }
  if (ir > JRATIO[24]) ir = JRATIO[24];
  if (ir > 1) {
    P->iratsh = ir;
    P->dvsc = double(ir) * dv_in;
    P->v1shft = double(ir - 1) * dv_in / 2.;
  } else {
    P->iratsh = 1;
    P->dvsc = dv_in;
    P->v1shft = 0.;
  }
  // CONVSC
  P->ratio = P->dvsc / P->dvo;
  const double dvodx = P->dvo / P->dxf, hwbnd = P->hwf / P->dvo;
  P->zslope = dvodx / hwhm;
  P->zbound = hwbnd * hwhm;
  P->xnorm = P->dvsc / hwhm;
  return LBL_OK;
}

}  // namespace lbl

namespace lbl {

void scnint_coefs(double* c) {
  const long NUMCOF = 201;
  const double XNUMCF = double(NUMCOF);
  for (long IP = 0; IP <= NUMCOF + 1; IP++) {
    const double P = (double(IP) - 1.0) / (XNUMCF - 1.0);
    const double PP = P * P;
    c[IP] = -P / 2.0 * ((1 - P) * (1 - P));
    c[203 + IP] = 1.0 - PP * (3.0 - 2.0 * P) + PP / 2.0 * (1.0 - P);
    c[406 + IP] = PP * (3.0 - 2.0 * P) + P / 2.0 * ((1.0 - P) * (1.0 - P));
    c[609 + IP] = -PP / 2 * (1.0 - P);
  }
}

// The host replay of INTERP's control flow (labels 20, 40, 80): the chunk
// bounds, the panel reads and, to decide them, each chunk's I and P
// carried point by point exactly as the kernel will carry them.
int scnint_plan(int64_t n, double v1_in, double dv_in, double dvo, std::vector<ScnChunk>* chunks,
                int64_t* n_fine, std::string* err) {
  chunks->clear();
  if (n < 2 || !(dv_in > 0.) || !(dvo > 0.)) {
    *err = "SCNINT: at least two input points and positive spacings";
    return LBL_E_ARG;
  }
  const double XNUMCF = 201.;
  const double V1 = v1_in;
  const long NUM = fint(((v1_in + double(n - 1) * dv_in - V1) / dvo) + 0.5);
  const double V2 = V1 + double(NUM) * dvo;
  const double DVI = dv_in, DVJ = dvo, VRATIO = DVJ / DVI;
  int64_t k = 0, nout = 0;
  double V1I = 0., V2I = 0.;
  long NNI = 0;
  bool eof = false;
  auto rdpanl = [&]() {
    const int64_t a = 2400 * k;
    if (a >= n) {
      eof = true;
      return;
    }
    const int64_t m = std::min<int64_t>(2400, n - a);
    V1I = (v1_in + double(a) * dv_in) - 4.0 * DVI;
    V2I = v1_in + double(a + m - 1) * dv_in;
    NNI = (long)m + 4;
    k++;
  };
  rdpanl();
  double V1J = V1, VJ = V1J;
  long J1 = 0, J2 = 0;
  auto emit = [&](long j1, long j2, int zero, long I, double P) {
    if (j2 < j1) return;
    ScnChunk c;
    c.out0 = nout + (j1 - 1);
    c.panel = k - 1;
    c.i0 = I;
    c.p0 = P;
    c.count = (int32_t)(j2 - j1 + 1);
    c.zero = zero;
    chunks->push_back(c);
  };
  auto panel_out = [&](long NNJ) {
    const double V2J = V1J + DVJ * double(NNJ - 1);
    nout += NNJ;
    V1J = V2J + DVJ;
  };
  while (V1J < V1I) {
    J2 = std::min<long>(fint((V1I - V1J) / DVJ) + 1, 2400);
    emit(1, J2, 1, 0, 0.);
    panel_out(J2);
    VJ = V1J;
  }
  for (long guard = 0;; guard++) {
    if (guard > 100000000L || (int64_t)chunks->size() > (int64_t(1) << 28)) {
      *err = "SCNINT: the interpolation makes no progress";
      return LBL_E_RANGE;
    }
    long I = fint((VJ - V1I) / DVI + 1.00001);
    const double VI = V1I + DVI * double(I - 1);
    double P = (VJ - VI) / DVI;
    J1 = fint((VJ - V1J) / DVJ + 1.001);
    J2 = std::min(std::min(fint((V2 - V1J) / DVJ + 1.001), fint((V2I - DVI - V1J) / DVJ + 1.)),
                  2400L);
    emit(J1, J2, 0, I, P);
    for (long J = J1; J <= J2; J++) {
      (void)fint(P * XNUMCF + 1.00001);
      P = P + VRATIO;
      if (P >= 1.0) {
        I = fint(double(I) + P);
        P = P - double(fint(P));
      }
    }
    VJ = V1J + DVJ * double(J2);
    if (J2 >= 2400 || VJ >= V2) {
      panel_out(J2);
      J2 = 0;
    }
    if (VJ >= V2) break;
    if (eof) {
      for (;;) {
        J1 = J2 + 1;
        J2 = std::min<long>(fint((V2 - V1J) / DVJ + 1.0001), 2400);
        emit(J1, J2, 1, 0, 0.);
        VJ = V1J + DVJ * double(J2);
        if (J2 >= 2400 || VJ >= V2) {
          panel_out(J2);
          J2 = 0;
        }
        if (!(VJ < V2)) break;
      }
      break;
    }
    if (I >= NNI - 2) {
      rdpanl();
      if (eof) V2I = V2I + DVI;
    }
  }
  *n_fine = nout;
  return LBL_OK;
}

}  // namespace lbl
