// lbl_kernels.cu -- sm_100a kernels of the layer optical-depth and merge path.
//
// Work is laid out on three global grids per layer instead of the
// reference's streamed 2400-point panels: R1 (spacing DV), R2 (4*DV) and R3
// (16*DV), all indexed from the panel-0 origin VFT0 = V1 - 32*DV with the
// reference's 1-based convention (grid point g sits at VFT0 + (g-1)*dv_k).
// A line's window limits are computed in panel-0 coordinates with Fortran
// truncation, which reproduces the reference for every panel (later panels
// only shift indices by multiples of 2400/600/150).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <type_traits>

#include "../data/cont_tables.h"
#include "../data/ref_tables.h"
#include "lbl_kernels.cuh"

namespace lbl {

namespace {

constexpr double kONEPL = 1.001, kONEMI = 0.999;
constexpr double kHWDXF = 4. / 0.002;        // HWF1/DXF1
constexpr double kODLO = 0.06;               // od_lo, src/lblparams.f90:47
constexpr int kChunk = 32;                   // far-wing lines decided per step

__constant__ double c_avrat[102], c_cf1[102], c_cf2[102], c_cf3[102], c_cgauss[102],
    c_cer[102];
__constant__ int c_isomax[48];

__device__ __forceinline__ long fint(double x) { return (long)x; }

// Radiation term (RADFN, src/oprop.f90:2235-2296)
__device__ double radfn(double vi, double xkt) {
  if (xkt > 0.0) {
    double x = vi / xkt;
    if (x <= 0.01) return 0.5 * x * vi;
    if (x <= 10.0) {
      double e = exp(-x);
      return vi * (1. - e) / (1. + e);
    }
  }
  return vi;
}

// Piecewise-linear radiation term over [VI, VINEW] (RADFNI, src/oprop.f90:2297-2475)
__device__ double radfni(double vi, double dvi, double xkt, double& vinew, double& rdel,
                         double& rdlast) {
  const double fact1 = 3.0E-03;
  const double xvi = vi;
  if (rdlast < 0.) rdlast = radfn(xvi, xkt);
  const double out = rdlast;
  long intvls = 1;
  double rdnext;
  double xviokt = xkt > 0.0 ? xvi / xkt : 0.;
  auto step = [&](double width) {
    if (vinew >= 0.0) {
      vinew = vi + width;
      intvls = fint((vinew - vi) / dvi);
      if (intvls < 1) intvls = 1;
      vinew = vi + dvi * double(intvls);
    } else {
      vinew = fabs(vinew);
      intvls = fint((vinew - vi) / dvi);
      if (intvls < 1) intvls = 1;
    }
  };
  if (xkt > 0.0 && xviokt <= 0.01) {
    step(fact1 * 0.5 * xvi);
    double xn = vinew / xkt;
    rdnext = 0.5 * xn * vinew;
  } else if (xkt > 0.0 && xviokt <= 10.0) {
    double e = exp(-xviokt);
    double xm = 1. - e, xp = 1. + e;
    double c = xviokt * e;
    step(fact1 * xvi / (1. + (c / xm + c / xp)));
    double en = exp(-(vinew / xkt));
    rdnext = vinew * (1. - en) / (1. + en);
  } else {
    step(fact1 * xvi);
    rdnext = vinew;
  }
  rdel = (rdnext - out) / double(intvls);
  rdlast = rdnext;
  return out;
}

// Planck function (PLANCK, src/xmerge.f90:968-1017) at XKT = T/RADCN2,
// with the exponent's argument VI/XKT taken as VI*rk (rk = RADCN2/T).
__device__ __forceinline__ double planck(double vi, double xkt, double rk) {
  double v = 0.;
  if (xkt > 0.0) {
    const double x = vi * rk;
    if (x < 1e-2) {
      v = (vi * vi) * xkt / (1. + 0.5 * x);
    } else if (x <= 80.) {
      const double e = exp(-x);
      v = (vi * vi * vi) * e / (1. - e);
    }
  }
  return v * kRADCN1;
}

__device__ __forceinline__ float bits_float(int32_t v) { return __int_as_float(v); }

// Y/G line-coupling coefficients carried by record i+1 (LNCOR1 :1039-1061,
// LINF4 :3163-3190).  upper=true selects LINF4's bracket convention.
__device__ void coupling(const DevLines& ln, int64_t i, int iflag, int ilc, double rectlc,
                         double tmpdif, bool linf4, double& yi, double& gi, double& g1,
                         double& g2) {
  double A[5], B[5];
  A[1] = ln.vraw[i + 1];
  B[1] = (double)ln.sp[i + 1];
  A[2] = (double)ln.alfa[i + 1];
  B[2] = (double)ln.epp[i + 1];
  A[3] = (double)bits_float(ln.mol[i + 1]);
  B[3] = (double)ln.hwhms[i + 1];
  A[4] = (double)ln.tmpalf[i + 1];
  B[4] = (double)ln.pshift[i + 1];
  double a, b;
  if (linf4) {
    double sa = (A[ilc] - A[ilc - 1]) * rectlc, sb = (B[ilc] - B[ilc - 1]) * rectlc;
    a = A[ilc] + sa * tmpdif;
    b = B[ilc] + sb * tmpdif;
  } else {
    double sa = (A[ilc + 1] - A[ilc]) * rectlc, sb = (B[ilc + 1] - B[ilc]) * rectlc;
    a = A[ilc] + sa * tmpdif;
    b = B[ilc] + sb * tmpdif;
  }
  if (iflag == 1) {
    yi = a;
    gi = b;
  } else {
    g1 = a;
    g2 = b;
  }
}

// air width with the O2/N2 foreign-width conversion of RDLIN/RDLNFL
__device__ __forceinline__ double air_width(const DevLines& ln, int64_t i, int m) {
  double a = (double)ln.alfa[i];
  if (m == 7) a = (a - 0.21 * (double)ln.hwhms[i]) / (1.0 - 0.21);
  if (m == 22) a = (a - 0.79 * (double)ln.hwhms[i]) / (1.0 - 0.79);
  return a;
}

// =========================================================================
// LINF4 line scaling (src/oprop.f90:3136-3220)
// =========================================================================
__global__ void k_far_scale(Work w, DevLines ln) {
  const int l = blockIdx.y;
  const LayerDev& L = w.L[l];
  const int64_t i = L.far_lo + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L.far_hi) return;
  const int64_t slot = L.off_far + (i - L.far_lo);
  int8_t ok = 0;
  if (ln.iflg[i] >= 0) {
    const int mcode = ln.mol[i];
    const int m = mcode % 100, iso = (mcode % 1000) / 100;
    if (m >= 1 && m <= 47 && iso >= 1 && iso <= c_isomax[m]) {
      const double wkm = (m <= L.nmol) ? L.wk[m] : 0.;
      double sui = (double)ln.sp[i] * wkm;
      const double vnu = ln.vnu[i];
      if (sui != 0. && vnu >= L.v1l4) {
        ok = 1;
        const int iflag = ln.iflg[i];
        double yi = 0., gi = 0., g1 = 0., g2 = 0.;
        if (iflag == 1 || iflag == 3)
          coupling(ln, i, iflag, L.ilc_f, L.rectlc_f, L.tmpdif_f, true, yi, gi, g1, g2);
        const double vs = vnu + L.rhorat * (double)ln.pshift[i];
        if (vs == 0.) sui = 2. * sui;
        double epp = (double)ln.epp[i];
        if (epp <= -1.001) epp = fabs(epp);
        if (epp > -0.999)
          sui = sui * L.scor[m][iso] * exp(-epp * L.betacr_f) * (1. + exp(-vs * L.beta_f));
        const double tmpcor = pow(L.tratio, (double)ln.tmpalf[i]);
        const double a0 = air_width(ln, i, m) * tmpcor;
        const double hs = (double)ln.hwhms[i] * tmpcor;
        double alfl = a0 * (L.rhorat - L.rhoslf[m]) + hs * L.rhoslf[m];
        if (iflag == 3) alfl = alfl * (1.0 - g1 * L.pavp0 - g2 * L.pavp2);
        w.f_vnu[slot] = vs;
        w.f_alfa[slot] = alfl;
        w.f_epp[slot] = vs * L.alfd1[m][iso];
        w.f_sp[slot] = sui * (1. + gi * L.pavp2);
        w.f_spp[slot] = sui * yi * L.pavp0;
        w.f_co2[slot] = (m == 2);
      }
    }
  }
  w.f_ok[slot] = ok;
}

// =========================================================================
// LINF4 segmenting + SHRINK (src/oprop.f90:3221-3292, 3508-3640): one thread
// per layer walks the TAPE3 panels in order.  Raw lines accumulate until at
// least LIMIN=1000 (shrunk-so-far + raw) are held, then the held raw lines
// are merged in groups of width DVR4/2 (non-CO2 and CO2 separately); a
// shrunk block is written once it holds >= 1000 lines or at the end.
// =========================================================================
// State of one SHRINK walk over raw far-wing lines in file order.
struct ShrinkWalk {
  double vlmt = 0.;
  bool started = false;
  bool pn = false, pc = false;  // the open group holds a line of positive strength
  double sal = 0., sad = 0., ss = 0., sv = 0.;      // open non-CO2 group (WRITE)
  double sal2 = 0., sad2 = 0., ss2 = 0., sv2 = 0.;  // open CO2 group (WRITE)
  int32_t raw = 0, out = 0;  // lines taken, shrunk lines written
};

// One layer's raw far-wing lines (LINF4 scaling) and shrunk-line outputs,
// indexed by 32-bit slot within the layer.
struct FarSlots {
  const int8_t *ok, *co2;
  const double *vnu, *sp, *spp, *alfa, *epp;
  double *s_vnu, *s_sp, *s_alfa, *s_epp, *s_spp;
  int8_t* s_co2;
};

__device__ __forceinline__ FarSlots far_slots(const Work& w, const LayerDev& L) {
  FarSlots f;
  const int64_t F = L.off_far, S = L.off_shr;
  f.ok = w.f_ok + F;
  f.co2 = w.f_co2 + F;
  f.vnu = w.f_vnu + F;
  f.sp = w.f_sp + F;
  f.spp = w.f_spp + F;
  f.alfa = w.f_alfa + F;
  f.epp = w.f_epp + F;
  f.s_vnu = w.s_vnu + S;
  f.s_sp = w.s_sp + S;
  f.s_alfa = w.s_alfa + S;
  f.s_epp = w.s_epp + S;
  f.s_spp = w.s_spp + S;
  f.s_co2 = w.s_co2 + S;
  return f;
}

// First usable raw line in slots [from, limit), searched by the whole warp
// 32 slots at a time; its centre in v.
__device__ bool next_valid_vnu(const FarSlots& fs, int32_t from, int32_t limit, double& v) {
  const int lane = threadIdx.x & 31;
  for (int32_t c = from; c < limit; c += 32) {
    const int32_t s = c + lane;
    const unsigned m = __ballot_sync(0xffffffffu, s < limit && fs.ok[s]);
    if (m) {
      v = __shfl_sync(0xffffffffu, s < limit ? fs.vnu[s] : 0., __ffs(m) - 1);
      return true;
    }
  }
  return false;
}

// SHRINK (src/oprop.f90:3508-3640) over slots [a, e) by one warp, 32
// slots at a time.  A group takes lines in file order while the next usable
// line (looked up before `limit`) lies within the group limit; the line
// where it does not closes the group and sets the next limit to its own
// centre + DVR4/2.  Non-CO2 and CO2 lines of a group are merged separately
// into strength-weighted lines (emitted when the group holds a line of
// positive strength); coupled lines pass through where they stand.
//   * closures: found in order with one ballot each against the limit the
//     previous closure set (warp-uniform state);
//   * sums (WRITE): the lane that ends a group adds its lines in file order
//     (the walk's own order), starting from the sums carried over from the
//     previous chunk when the group began there;
//   * outputs: every lane's count (coupled line, group lines) is prefix-
//     summed over the warp, so the shrunk lines land in walk order at
//     shrunk slot `out`.
template <bool WRITE>
__device__ void shrink_walk(const FarSlots& fs, const LayerDev& L, int32_t a, int32_t e,
                            int32_t limit, ShrinkWalk& st) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const double dvh = L.dvr4 / 2.;
  for (int32_t c = a; c < e; c += 32) {
    const int32_t s = c + lane;
    const bool valid = s < e && fs.ok[s];
    double v = 0., sp = 0., spp = 0., al = 0., ep = 0.;
    int co2 = 0;
    if (valid) {
      v = fs.vnu[s];
      sp = fs.sp[s];
      spp = fs.spp[s];
      if (sp < 1.0e-35) {
        sp = 0.;
        spp = 0.;
      }
      co2 = fs.co2[s];
      if (WRITE) {
        al = fs.alfa[s];
        ep = fs.epp[s];
      }
    }
    const unsigned m = __ballot_sync(full, valid);
    if (!m) continue;
    const int first = __ffs(m) - 1, last = 31 - __clz(m);
    // centre of the next usable line (after the chunk for the last lane)
    const unsigned up = m & ~(below | (1u << lane));
    double vn = __shfl_sync(full, v, up ? __ffs(up) - 1 : lane);
    bool hn = up != 0;
    double vx = 0.;
    const bool hx = next_valid_vnu(fs, (c + 32 < e) ? c + 32 : e, limit, vx);
    if (lane == last) {
      hn = hx;
      vn = vx;
    }
    if (!st.started) {
      st.vlmt = __shfl_sync(full, v, first) + dvh;
      st.started = true;
    }
    st.raw += __popc(m);
    // Where the chunk's centres do not decrease, a line whose next usable
    // line lies beyond its own centre + DVR4/2 closes its group under any
    // limit set inside the chunk (such a limit is at most that bound), so
    // after a closure a run of such lines closes in one step.
    const unsigned forced = __ballot_sync(full, valid && !(hn && vn <= v + dvh));
    const bool sorted = __ballot_sync(full, valid && hn && lane != last && vn < v) == 0u;
    unsigned cl = 0;  // lanes that close a group
    for (int pos = first; pos <= last;) {
      const unsigned q = __ballot_sync(full, valid && lane >= pos && !(hn && vn <= st.vlmt));
      if (!q) break;
      int k = __ffs(q) - 1;
      cl |= 1u << k;
      if (sorted) {
        const unsigned after = m & ~((2u << k) - 1u);  // usable lanes above k
        const unsigned nf = after & ~forced;
        const unsigned run = nf ? (after & ((1u << (__ffs(nf) - 1)) - 1u)) : after;
        if (run) {
          cl |= run;
          k = 31 - __clz(run);
        }
      }
      st.vlmt = __shfl_sync(full, v, k) + dvh;
      pos = k + 1;
    }
    const bool cpl = valid && spp != 0.;
    const unsigned mN = __ballot_sync(full, valid && !cpl && !co2 && sp > 0.);
    const unsigned mC = __ballot_sync(full, valid && !cpl && co2 && sp > 0.);
    const bool isc = (cl >> lane) & 1u;
    const bool ends = isc || (lane == last);  // a closure or the chunk's open tail
    const unsigned prevs = cl & below;
    const int gs = prevs ? 32 - __clz(prevs) : 0;  // first lane of this lane's group
    const unsigned rng = (lane == 31 ? full : ((2u << lane) - 1u)) & ~((1u << gs) - 1u);
    const bool carry = prevs == 0;  // the group began before this chunk
    const bool gN = ends && (((mN & rng) != 0u) || (carry && st.pn));
    const bool gC = ends && (((mC & rng) != 0u) || (carry && st.pc));
    const int ec = (cpl ? 1 : 0) + (isc ? (gN ? 1 : 0) + (gC ? 1 : 0) : 0);
    const unsigned b0 = __ballot_sync(full, ec & 1), b1 = __ballot_sync(full, ec & 2);
    const bool open = !((cl >> last) & 1u);
    if (WRITE) {
      double sv = 0., ss = 0., sal = 0., sad = 0., sv2 = 0., ss2 = 0., sal2 = 0., sad2 = 0.;
      if (ends && carry) {
        sv = st.sv; ss = st.ss; sal = st.sal; sad = st.sad;
        sv2 = st.sv2; ss2 = st.ss2; sal2 = st.sal2; sad2 = st.sad2;
      }
      const int len = ends ? lane - gs + 1 : 0;
      const int maxlen = __reduce_max_sync(full, (unsigned)len);
      const int kind = (valid && !cpl) ? (co2 ? 2 : 1) : 0;
      for (int t = 0; t < maxlen; t++) {
        const int src = (gs + t) & 31;
        const double vi = __shfl_sync(full, v, src);
        const double spi = __shfl_sync(full, sp, src);
        const double ali = __shfl_sync(full, al, src);
        const double epi = __shfl_sync(full, ep, src);
        const int ki = __shfl_sync(full, kind, src);
        if (t < len) {
          if (ki == 1) {
            sv = sv + vi * spi;
            ss = ss + spi;
            sal = sal + spi * ali;
            sad = sad + spi * epi;
          } else if (ki == 2) {
            sv2 = sv2 + vi * spi;
            ss2 = ss2 + spi;
            sal2 = sal2 + spi * ali;
            sad2 = sad2 + spi * epi;
          }
        }
      }
      int o = st.out + __popc(b0 & below) + 2 * __popc(b1 & below);
      auto put = [&](double vnu, double spv, double alfa, double epp, double sppv, int c2) {
        fs.s_vnu[o] = vnu;
        fs.s_sp[o] = spv;
        fs.s_alfa[o] = alfa;
        fs.s_epp[o] = epp;
        fs.s_spp[o] = sppv;
        fs.s_co2[o] = (int8_t)c2;
        o++;
      };
      if (cpl) put(v, sp, al, ep, spp, co2);
      if (isc && gN) put(sv / ss, ss, sal / ss, sad / ss, 0., 0);
      if (isc && gC) put(sv2 / ss2, ss2, sal2 / ss2, sad2 / ss2, 0., 1);
      st.sv = open ? __shfl_sync(full, sv, last) : 0.;
      st.ss = open ? __shfl_sync(full, ss, last) : 0.;
      st.sal = open ? __shfl_sync(full, sal, last) : 0.;
      st.sad = open ? __shfl_sync(full, sad, last) : 0.;
      st.sv2 = open ? __shfl_sync(full, sv2, last) : 0.;
      st.ss2 = open ? __shfl_sync(full, ss2, last) : 0.;
      st.sal2 = open ? __shfl_sync(full, sal2, last) : 0.;
      st.sad2 = open ? __shfl_sync(full, sad2, last) : 0.;
    }
    st.out += __popc(b0) + 2 * __popc(b1);
    const bool pn = __shfl_sync(full, gN, last), pc = __shfl_sync(full, gC, last);
    st.pn = open && pn;
    st.pc = open && pc;
  }
}

// Parallel form of the LINF4 panel loop.  A segment (the raw lines held
// between two SHRINK calls) always starts at a TAPE3 panel boundary and ends
// at the first panel end where held-shrunk + raw >= LIMIN, so:
//   k_shr_count  for every start panel b, walks forward and records the raw
//                count and the shrunk-output count a segment b..e would have;
//   k_shr_plan   per layer, replays the LINF4 state machine on those counts
//                (segments, their output offsets, shrunk-block starts);
//   k_shr_write  per segment, performs SHRINK and writes the shrunk lines.
__device__ __forceinline__ int64_t far_slot_begin(const LayerDev& L, const int64_t* bs, int64_t b) {
  return bs[b] > L.far_lo ? bs[b] - L.far_lo : 0;
}
__device__ __forceinline__ int64_t far_slot_end(const LayerDev& L, const int64_t* bs, int64_t b) {
  const int64_t e = bs[b + 1] - L.far_lo;
  const int64_t n = L.far_hi - L.far_lo;
  return e > n ? n : e;
}

// One warp per (layer, start block).
__global__ void k_shr_count(Work w, const int64_t* bs, const int64_t* blk_base, int nlay) {
  const int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  // warp -> (layer, local start block) through the per-layer block base
  int lo = 0, hi = nlay;
  while (lo < hi) {
    int m = (lo + hi) >> 1;
    if (blk_base[m + 1] <= t) lo = m + 1;
    else hi = m;
  }
  if (lo >= nlay) return;
  const int l = lo;
  const LayerDev& L = w.L[l];
  const int64_t bl = t - blk_base[l];
  const int64_t nb = L.fblk_hi - L.fblk_lo;
  if (bl >= nb) return;
  int32_t* craw = w.c_raw + (blk_base[l] + bl) * kSegMaxBlk;
  int32_t* cout = w.c_out + (blk_base[l] + bl) * kSegMaxBlk;
  const int32_t nfar = (int32_t)(L.far_hi - L.far_lo);
  const FarSlots fs = far_slots(w, L);
  ShrinkWalk st;
  int k = 0;
  for (int64_t b = L.fblk_lo + bl; b < L.fblk_hi && k < kSegMaxBlk; b++, k++) {
    shrink_walk<false>(fs, L, (int32_t)far_slot_begin(L, bs, b), (int32_t)far_slot_end(L, bs, b),
                       nfar, st);
    // the segment's raw and output counts were it closed at this block's end
    if (lane == 0) {
      craw[k] = (int32_t)st.raw;
      cout[k] = (int32_t)(st.out + (st.pn ? 1 : 0) + (st.pc ? 1 : 0));
    }
    if (st.raw >= 1000) {
      k++;
      break;
    }
  }
  if (lane == 0)
    for (; k < kSegMaxBlk; k++) craw[k] = -1;  // not reached
}

// One warp per layer: the LINF4 state machine over the count tables, the
// end of each segment found by one ballot over its start panel's row.
__global__ void k_shr_plan(Work w, const int64_t* blk_base) {
  const int l = blockIdx.x;
  const int lane = threadIdx.x;
  const unsigned full = 0xffffffffu;
  if (l >= w.nlay) return;
  const LayerDev& L = w.L[l];
  int64_t nseg = 0, total = 0, nb9 = 0, blk_start = 0, J = 0;
  static_assert(kSegMaxBlk <= 64, "two entries of a count row per lane");
  if (L.ilblf4 >= 1 && L.far_hi > L.far_lo) {
    const int64_t nb = L.fblk_hi - L.fblk_lo;
    int64_t b = 0;
    while (b < nb) {
      const int32_t* craw = w.c_raw + (blk_base[l] + b) * kSegMaxBlk;
      const int32_t* cout = w.c_out + (blk_base[l] + b) * kSegMaxBlk;
      // segment b..b+k ends at the first k reaching the last panel or
      // holding + raw >= 1000; an unreached entry (-1) or k past the row
      // means the segment is longer than the table
      const int k0 = lane, k1 = lane + 32;
      const int32_t r0 = craw[k0], r1 = k1 < kSegMaxBlk ? craw[k1] : -1;
      const bool h0 = r0 < 0 || b + k0 == nb - 1 || J + r0 >= 1000;
      const bool h1 = r1 < 0 || b + k1 == nb - 1 || J + r1 >= 1000;
      const unsigned m0 = __ballot_sync(full, h0), m1 = __ballot_sync(full, h1);
      const int k = m0 ? __ffs(m0) - 1 : (m1 ? 32 + __ffs(m1) - 1 : 64);
      const int32_t rk = k < 32 ? __shfl_sync(full, r0, k & 31) : __shfl_sync(full, r1, k & 31);
      if (k >= kSegMaxBlk || rk < 0) {
        if (lane == 0) {
          w.status[0] = 2;  // segment longer than the count table: fall back
          w.s_count[l] = -1;
        }
        return;
      }
      const int64_t n = cout[k];
      if (lane == 0) {
        w.seg_blk[L.off_seg + nseg] = (int32_t)b;
        w.seg_nblk[L.off_seg + nseg] = (int32_t)(k + 1);
        w.seg_out[L.off_seg + nseg] = total;
      }
      nseg++;
      total += n;
      J += n;
      b += k + 1;
      if (J >= 1000 || b >= nb) {
        if (J > 0) {
          if (lane == 0) w.b9_start[L.off_blk9 + nb9] = blk_start;
          nb9++;
        }
        blk_start = total;
        J = 0;
      }
    }
  }
  if (lane == 0) {
    w.seg_count[l] = nseg;
    w.s_count[l] = total;
    w.b9_count[l] = nb9;
  }
}

// One warp per segment.
__global__ void k_shr_write(Work w, const int64_t* bs, const int64_t* seg_base, int nlay) {
  const int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lo = 0, hi = nlay;
  while (lo < hi) {
    int m = (lo + hi) >> 1;
    if (seg_base[m + 1] <= t) lo = m + 1;
    else hi = m;
  }
  if (lo >= nlay) return;
  const int l = lo;
  const LayerDev& L = w.L[l];
  const int64_t sgi = t - seg_base[l];
  if (w.s_count[l] < 0 || sgi >= w.seg_count[l]) return;
  const int64_t b0 = L.fblk_lo + w.seg_blk[L.off_seg + sgi];
  const int64_t b1 = b0 + w.seg_nblk[L.off_seg + sgi];
  ShrinkWalk st;
  st.out = (int32_t)w.seg_out[L.off_seg + sgi];
  const int32_t e = (int32_t)far_slot_end(L, bs, b1 - 1);
  shrink_walk<true>(far_slots(w, L), L, (int32_t)far_slot_begin(L, bs, b0), e, e, st);
}

// =========================================================================
// LBLF4/CONVF4 far wing (src/oprop.f90:3641-4039), one CTA per window.
// Lines are taken in file order 32 at a time; one warp decides acceptance
// exactly as the reference's in-order test against the partially
// accumulated R4 while the other threads add the previously accepted lines
// to the window points they own (see k_far_wing).
// =========================================================================

// FP32 evaluation constants of one side (line or image) of a line.  The
// offset from the line centre and the distance to the bound B are taken
// from integer point offsets plus fractions fixed per line in FP64:
//     x_j     = (j - jc) dv - dlt
//     B - x_j = ((mp - (j - jc)) + php) dv      (x_j >= 0)
//     B + x_j = ((mm + (j - jc)) + phm) dv      (x_j <  0)
// so u = B - |x_j| keeps its relative precision as x_j approaches B.
struct F4Side32 {
  float dlt, php, phm, mpf, mmf, dptrat;
  int32_t jc;
};

struct F4Line64 {
  // FP64 constants (CONVF4 :3965-3986); dptrat is 0 for an uncoupled line
  double xnui, sil, siv_a3, siv_b3, alfl2, rvi2, f4bnd, dptrat, mxnui, mdptrat;
  int32_t jmin, jmax, mjmin, mjmax, co2, has;  // has: 1 line, 2 image; empty range if absent
};
// with the FP32 copies for split-precision evaluation
struct F4Line : F4Line64 {
  float sil32, sa3_32, sb3_32, alfl2_32, rvi2_32, f4bnd32, rdd32;  // rdd = F4BND/B^2
  F4Side32 s32[2];
};

// Reciprocal from the hardware estimate (rcp.approx) refined by
// Newton-Raphson steps r <- r + r (1 - x r), each of which squares the
// relative error: two steps take the FP64 estimate to full precision, one
// step the FP32 estimate.  Used for the per-point divisions of the far wing,
// whose denominators alpha^2 + x^2 are positive and normal.
__device__ __forceinline__ double recip_nr(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  double e = fma(-x, r, 1.);
  r = fma(r, e, r);
  e = fma(-x, r, 1.);
  return fma(r, e, r);
}
__device__ __forceinline__ float recip_nr(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return fmaf(r, fmaf(-x, r, 1.f), r);
}

// F4 of one side of line q at window point j in FP64 (CONVF4 :3990-4009);
// 0 outside the side's point range.  Branch-free apart from the range, so
// that several lines evaluate together.
__device__ __forceinline__ double f4_side(const F4Line64& q, bool image, int j, double dvr4,
                                          double rbndsq) {
  const double xnui = image ? q.mxnui : q.xnui;
  const int lo = image ? q.mjmin : q.jmin, hi = image ? q.mjmax : q.jmax;
  const double xm = double(j - 1) * dvr4 - xnui;
  const double xmsq = xm * xm;
  const double zvsq = xmsq * q.rvi2;
  const double sub = q.co2 ? (2. - xmsq * rbndsq) * q.f4bnd : q.f4bnd;
  double f = zvsq <= 4096. ? (q.siv_a3 + zvsq * q.siv_b3) - sub
                           : q.sil * recip_nr(q.alfl2 + xmsq) - sub;
  f = f + xm * (image ? q.mdptrat : q.dptrat) * f;
  return (j >= lo && j <= hi) ? f : 0.;
}

// One side of a line held in an adder's registers.
template <typename T>
struct F4Reg;

template <>
struct F4Reg<double> {
  double sil, sa3, sb3, alfl2, rvi2, f4bnd, dptrat, xnui;
  int co2;
};

template <>
struct F4Reg<float> {
  float sil, sa3, sb3, alfl2, rvi2, f4bnd, rdd, dptrat, dlt, php, phm, mpf, mmf, k0;
  int co2;
};

__device__ __forceinline__ void f4_load(F4Reg<double>& r, const F4Line64& p, int m, int) {
  r.sil = p.sil;
  r.sa3 = p.siv_a3;
  r.sb3 = p.siv_b3;
  r.alfl2 = p.alfl2;
  r.rvi2 = p.rvi2;
  r.f4bnd = p.f4bnd;
  r.dptrat = m ? p.mdptrat : p.dptrat;
  r.xnui = m ? p.mxnui : p.xnui;
  r.co2 = p.co2;
}

// j0: the adder's first window point; k0 = j0 - jc is a float so that
// j - jc at the adder's later points is an exact float sum.
__device__ __forceinline__ void f4_load(F4Reg<float>& r, const F4Line& p, int m, int j0) {
  const F4Side32& sd = p.s32[m];
  r.sil = p.sil32;
  r.sa3 = p.sa3_32;
  r.sb3 = p.sb3_32;
  r.alfl2 = p.alfl2_32;
  r.rvi2 = p.rvi2_32;
  r.f4bnd = p.f4bnd32;
  r.rdd = p.rdd32;
  r.dptrat = sd.dptrat;
  r.dlt = sd.dlt;
  r.php = sd.php;
  r.phm = sd.phm;
  r.mpf = sd.mpf;
  r.mmf = sd.mmf;
  r.k0 = (float)(j0 - sd.jc);
  r.co2 = p.co2;
}

// F4 at window point j = j0 + kq - k0 (FP32).  Beyond the quadratic core
// the bound is subtracted without cancellation, with v = B^2 - x^2 = u (2B - u):
//   non-CO2  L(x) - L(B)               =  F4BND v / (a^2 + x^2)
//   CO2      L(x) - (2 - x^2/B^2) L(B) =  (F4BND/B^2) v (v - a^2) / (a^2 + x^2)
__device__ __forceinline__ float f4_at(const F4Reg<float>& r, int, float kq, double, double,
                                       float dvr4f, float bndf, float rbndsqf) {
  const float xm = kq * dvr4f - r.dlt;
  const float xmsq = xm * xm;
  const float zvsq = xmsq * r.rvi2;
  float f;
  if (zvsq <= 4096.f) {
    const float sub = r.co2 ? (2.f - xmsq * rbndsqf) * r.f4bnd : r.f4bnd;
    f = (r.sa3 + zvsq * r.sb3) - sub;
  } else {
    const float u = (xm >= 0.f ? (r.mpf - kq) + r.php : (r.mmf + kq) + r.phm) * dvr4f;
    const float v = u * (2.f * bndf - u);
    const float rden = recip_nr(r.alfl2 + xmsq);
    f = r.co2 ? (r.rdd * v) * (v - r.alfl2) * rden : (r.f4bnd * v) * rden;
  }
  return f + xm * r.dptrat * f;
}

// A far-wing CTA is one deciding warp plus ADDERS threads that own the
// window's points (point j belongs to adder (j-1) % ADDERS).
constexpr int kFwSmem = 2 * (int)kR4Stride * (int)sizeof(double);  // two R4 buffers
// split precision adds one FP32 accumulator per adder point
constexpr int fw_smem32(int adders) {
  return kFwSmem + ((kLimOut + adders - 1) / adders) * adders * (int)sizeof(float);
}
// Barrier of the DEC deciding warps only (named barrier 1); the adders never
// take part in it.
template <int DEC>
__device__ __forceinline__ void fw_dec_sync() {
  asm volatile("bar.sync 1, %0;" ::"r"(DEC * 32) : "memory");
}

// The CTA works in phases separated by one barrier.  In phase t the deciding
// warps take chunk t (32 consecutive lines of the layer's shrunk list) and
// decide every line exactly as CONVF4's in-order test against the partial
// R4 at its point JJ, where that partial R4 is
//     R4 through chunk t-2   (buffer written in phase t-1)
//   + chunk t-1's accepted lines, evaluated at JJ directly
//   + the earlier accepted lines of chunk t, evaluated at JJ directly;
// meanwhile the adders evaluate chunk t-1's accepted lines over the whole
// window and write R4 through chunk t-1 into the other buffer.  The deciding
// warps split the direct evaluations (up to 32 x 32 line-point pairs for each
// of the two chunks) among themselves; warp 0 then sums each line's terms in
// CONVF4's order.  The in-chunk order dependence is resolved speculatively:
// every line is first decided against the lines accepted on their own
// partial R4 alone; the lowest line whose decision differs from that guess is
// exact, so the guess is corrected there and the lines above it re-decided,
// until no line differs.
//
// ADDERS and DEC (deciding warps) set the CTA's width; the autotuner picks
// among the variants.
template <typename T, int ADDERS, int DEC, int MINB>
__global__ void __launch_bounds__(ADDERS + 32 * DEC, MINB)
    k_far_wing(Work w, const int32_t* win_order, const int32_t* win_layer) {
  constexpr int kFwAdders = ADDERS;
  constexpr int kFwThreads = ADDERS + 32 * DEC;
  static_assert(DEC >= 2, "warp 1 builds the line constants");
  constexpr int kFwPts = (kLimOut + ADDERS - 1) / ADDERS;  // window points per adder
  extern __shared__ double fw_r4[];  // [2][kR4Stride]
  // FP64 line constants (and the FP32 copies in split precision) of chunks
  // t-1, t and t+1, and what the decisions need of each line
  using Line = typename std::conditional<sizeof(T) == 8, F4Line64, F4Line>::type;
  __shared__ Line cl[3][kChunk];
  __shared__ double s_speak[3][kChunk], s_vnu[3][kChunk], s_spp[3][kChunk];
  __shared__ int s_jj[3][kChunk];
  __shared__ unsigned s_okm[3];
  __shared__ unsigned s_imgc[3];  // lines of the chunk with a Van Vleck-Weisskopf image
  __shared__ unsigned s_imgp[3];  // the same of the accepted lines, in s_idx order
  __shared__ int s_nval[3];  // lines in the chunk (0: none)
  __shared__ int s_idx[3][kChunk];
  __shared__ int s_nacc[3];
  __shared__ int s_state[2];  // by phase parity: a chunk was decided
  __shared__ int s_stop;      // a decided line ended the window
  __shared__ double s_x[kChunk][kChunk];  // chunk t-1's lines at chunk t's points
  __shared__ double s_y[kChunk][kChunk];  // chunk t at its own points (line; image)
  __shared__ unsigned s_lm;
  const int gw = win_order[blockIdx.x];
  const int l = win_layer[gw];
  const LayerDev& L = w.L[l];
  const WinDev& W = w.win[gw];
  for (int j = threadIdx.x; j < 2 * kR4Stride; j += kFwThreads) fw_r4[j] = 0.;
  if constexpr (sizeof(T) == 4) {
    float* acc32 = reinterpret_cast<float*>(fw_r4 + 2 * kR4Stride);
    for (int j = threadIdx.x; j < kFwPts * kFwAdders; j += kFwThreads) acc32[j] = 0.f;
  }
  const double dvr4 = L.dvr4, bnd = L.bound4, bndsq = bnd * bnd, rbndsq = 1. / bndsq;
  const int npt = W.nptr4;
  const int64_t S = L.off_shr;
  const int64_t ns = w.s_count[l];
  const int64_t nb9 = w.b9_count[l];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned full = 0xffffffffu;
  // The line stream: warp 1 walks the layer's shrunk list (TAPE9 blocks, 32
  // lines a chunk), building each chunk's line constants one phase ahead of
  // warp 0's decisions.
  int64_t b = -1, c0 = 0, b1 = 0;
  bool dmore = false;
  auto next_block = [&]() {
    for (b = b + 1; b < nb9; b++) {
      c0 = w.b9_start[L.off_blk9 + b];
      b1 = (b + 1 < nb9) ? w.b9_start[L.off_blk9 + b + 1] : ns;
      if (!(w.s_vnu[S + b1 - 1] < W.vlo)) return true;  // RDLIN4 skips VMAX < VLO (:3815)
    }
    return false;
  };
  // raw values of warp 1's next line, loaded one phase ahead
  double n_sp = 0., n_spp = 0., n_ad = 0., n_al = 0., n_v = 0.;
  int n_co2 = 0;
  auto prefetch = [&]() {
    const int64_t i = c0 + lane;
    if (dmore && i < b1) {
      n_sp = w.s_sp[S + i];
      n_spp = w.s_spp[S + i];
      n_ad = w.s_epp[S + i];
      n_al = w.s_alfa[S + i];
      n_v = w.s_vnu[S + i];
      n_co2 = w.s_co2[S + i];
    }
  };
  // Warp 1: the chunk at c0 into buffer k (one line per lane, CONVF4
  // :3965-3986), then on to the next chunk, whose raw values it prefetches.
  auto build = [&](int k) {
    const int64_t i = c0 + lane;
    Line& p = cl[k][lane];
    p.has = 0;
    bool ok = false;
    double speak = 0., vnu = 0., spp = 0.;
    int jj = 1, has = 0;
    if (dmore && i < b1) {
        const double recpi = 1. / (2. * asin(1.));
        const double zsq = 64. * 64.;
        const double A3 = (1. + 2. * zsq) / ((1. + zsq) * (1. + zsq));
        const double B3 = -1. / ((1. + zsq) * (1. + zsq));
        const double sp = n_sp;
        spp = n_spp;
        ok = !(sp == 0. && spp == 0.);
        const double ad = n_ad, al = n_al, v = n_v;
        const double zeta = al / (al + ad);
        long iz = fint(100. * zeta + kONEPL);
        iz = iz < 1 ? 1 : (iz > 101 ? 101 : iz);  // zeta in [0,1]; guards bad input
        const double zd = 100. * zeta - double(iz - 1);
        const double alfav =
            (c_avrat[iz - 1] + zd * (c_avrat[iz] - c_avrat[iz - 1])) * (al + ad);
        const double ralfv = 1. / alfav;
        const double sil = sp * recpi * al;
        const double siv = (al * ralfv) * sp * recpi * ralfv;
        speak = A3 * fabs(siv);
        long jjl = fint((v - W.v1r4) / dvr4 + 1.);
        jjl = jjl < 1 ? 1 : (jjl > npt ? npt : jjl);
        jj = (int)jjl;
        vnu = v;
        const double dptrat = spp != 0. ? spp / (sp * alfav) : 0.;
        p.xnui = v - W.v1r4;
        p.sil = sil;
        p.siv_a3 = siv * A3;
        p.siv_b3 = siv * B3;
        p.alfl2 = al * al;
        p.rvi2 = 1. / (alfav * alfav);
        p.f4bnd = sil / (al * al + bndsq);
        p.dptrat = dptrat;
        p.co2 = n_co2;
        const long jmin = fint((p.xnui - bnd) / dvr4 + 2.);
        const long jmax = fint((p.xnui + bnd) / dvr4 + 1.);
        const bool beyond = jmin > npt;  // GO TO 60: no wing, no image
        p.jmin = (int)(jmin < 1 ? 1 : jmin);
        p.jmax = (int)(jmax > npt ? npt : jmax);
        if (beyond || p.jmax < p.jmin) p.jmin = 1, p.jmax = 0;
        else p.has |= 1;
        p.mxnui = -v - W.v1r4;
        p.mdptrat = -dptrat;
        p.mjmin = 1;
        p.mjmax = 0;
        if (!beyond && v > 0. && v <= 25.) {  // Van Vleck-Weisskopf image (:4014-4024)
          const long mjmin = fint((p.mxnui - bnd) / dvr4 + 2.);
          const long mjmax = fint((p.mxnui + bnd) / dvr4 + 1.);
          if (mjmin <= npt && (mjmax > npt ? npt : mjmax) >= (mjmin < 1 ? 1 : mjmin)) {
            p.mjmin = (int)(mjmin < 1 ? 1 : mjmin);
            p.mjmax = (int)(mjmax > npt ? npt : mjmax);
            p.has |= 2;
          }
        }
        has = p.has;
        if constexpr (sizeof(T) == 4) {
          p.sil32 = (float)p.sil;
          p.sa3_32 = (float)p.siv_a3;
          p.sb3_32 = (float)p.siv_b3;
          p.alfl2_32 = (float)p.alfl2;
          p.rvi2_32 = (float)p.rvi2;
          p.f4bnd32 = (float)p.f4bnd;
          p.rdd32 = (float)(p.f4bnd * rbndsq);
          const double rdv = 1. / dvr4;
  #pragma unroll
          for (int m = 0; m < 2; m++) {
            if (!(has & (1 << m))) continue;
            F4Side32& sd = p.s32[m];
            const double xn = m ? p.mxnui : p.xnui;
            const double jc = floor(xn * rdv + 1.5);
            const double dl = xn - (jc - 1.) * dvr4;
            const double tp = (bnd + dl) * rdv, tm = (bnd - dl) * rdv;
            const double mp = floor(tp), mm = floor(tm);
            sd.jc = (int32_t)jc;
            sd.dlt = (float)dl;
            sd.php = (float)(tp - mp);
            sd.phm = (float)(tm - mm);
            sd.mpf = (float)mp;
            sd.mmf = (float)mm;
            sd.dptrat = (float)(m ? p.mdptrat : p.dptrat);
          }
        }
    }
    (void)has;
    s_speak[k][lane] = speak;
    s_vnu[k][lane] = vnu;
    s_spp[k][lane] = spp;
    s_jj[k][lane] = jj;
    const unsigned okm = __ballot_sync(0xffffffffu, ok);
    const unsigned imgc = __ballot_sync(0xffffffffu, (p.has & 2) != 0);
    if (lane == 0) {
      s_okm[k] = okm;
      s_imgc[k] = imgc;
      s_nval[k] = dmore ? (int)((b1 - c0) < kChunk ? (b1 - c0) : kChunk) : 0;
    }
    if (dmore) {
      c0 += kChunk;
      if (c0 >= b1) dmore = next_block();
      prefetch();
    }
  };
  if (warp == 1) {
    dmore = next_block();
    prefetch();
    build(0);
  }
  if (threadIdx.x == 0) s_stop = 0;
  __syncthreads();
  int rb = 0;      // buffer holding R4 through chunk t-2 in phase t
  int cur = 0;     // line buffer of chunk t (chunk t-1 and t+1 in the others)
  bool have_prev = false;
  unsigned long long nevals = 0;
  for (int ph = 0;; ph++) {
    const double* R4r = fw_r4 + rb * kR4Stride;
    double* R4w = fw_r4 + (rb ^ 1) * kR4Stride;
    const int prv = cur == 0 ? 2 : cur - 1;  // chunk t-1
    const int nxt = cur == 2 ? 0 : cur + 1;  // chunk t+1
    if (warp < DEC) {
      // chunk t exists and no earlier line ended the window
      const bool go = s_nval[cur] > 0 && !s_stop;
      // Stage 1: the deciding warps evaluate chunk t-1's accepted lines at
      // every line's point JJ (s_x; their Van Vleck-Weisskopf images, rare,
      // are evaluated in stage 2).
      if (go) {
        const int jjb = s_jj[cur][lane];
        const int np = have_prev ? s_nacc[prv] : 0;
#pragma unroll 2
        for (int a = warp; a < np; a += DEC)
          s_x[a][lane] = f4_side(cl[prv][s_idx[prv][a]], false, jjb, dvr4, rbndsq);
      }
      fw_dec_sync<DEC>();
      // Stage 2: warp 0 completes each line's partial R4 through chunk t-1
      // in CONVF4's order and guesses the lines accepted on it alone (live).
      bool ok = false, live = false;
      double speak = 0., r = 0., vnu = 0., spp = 0.;
      int jj = 1, has = 0;
      const double dptmn = W.dptmn, dptfc = L.dptfc;
      if (warp == 0 && go) {
        ok = (s_okm[cur] >> lane) & 1u;
        speak = s_speak[cur][lane];
        vnu = s_vnu[cur][lane];
        spp = s_spp[cur][lane];
        jj = s_jj[cur][lane];
        has = cl[cur][lane].has;
        if (ok) r = R4r[jj];
        const int np = have_prev ? s_nacc[prv] : 0;
        if (ok) {
          // (adding an absent image's 0 would leave r unchanged: r is never -0)
          const unsigned imgp = have_prev ? s_imgp[prv] : 0u;
          for (int a = 0; a < np; a++) {
            r += s_x[a][lane];
            if ((imgp >> a) & 1u) r += f4_side(cl[prv][s_idx[prv][a]], true, jj, dvr4, rbndsq);
          }
        }
        live = ok && !(speak <= (dptmn + dptfc * r) && spp == 0.);
        const unsigned lm = __ballot_sync(full, live);
        if (lane == 0) s_lm = lm;
      }
      fw_dec_sync<DEC>();
      // Stage 3: the deciding warps evaluate the live lines of chunk t at the
      // points of the lines above them (s_y[a][b]: line a at b's point; its
      // image at s_y[b][a]), the live lines shared out in turn.
      if (go) {
        const int jjb = s_jj[cur][lane];
        const int nv = s_nval[cur];
        const unsigned imgc = s_imgc[cur];
        int k = 0;
        for (unsigned m = s_lm; m; m &= m - 1, k++) {
          const int a = __ffs(m) - 1;
          if (k % DEC != warp) continue;
          if (lane > a && lane < nv) {
            const Line& q = cl[cur][a];
            s_y[a][lane] = f4_side(q, false, jjb, dvr4, rbndsq);
            s_y[lane][a] = ((imgc >> a) & 1u) ? f4_side(q, true, jjb, dvr4, rbndsq) : 0.;
          }
        }
      }
      fw_dec_sync<DEC>();
      // Stage 4: warp 0 decides chunk t while warp 1 builds chunk t+1 (used
      // only if no line of chunk t ends the window).
      if (warp == 0) {
        int decided = 0;
        if (go) {
          const unsigned lm = s_lm;
          // earlier lines of this chunk accepted on their own partial R4
          double part = r;  // continues the running sum in CONVF4's order
          const unsigned imgc = s_imgc[cur];
          if (ok) {
            for (unsigned m = lm & ((1u << lane) - 1u); m; m &= m - 1) {
              const int a = __ffs(m) - 1;
              part += s_y[a][lane];
              if ((imgc >> a) & 1u) part += s_y[lane][a];
            }
          }
          bool acc = ok && !(speak <= (dptmn + dptfc * part) && spp == 0.);
          unsigned mis = __ballot_sync(full, acc != live);
          while (mis) {
            const int f = __ffs(mis) - 1;  // every line below f is decided exactly
            const bool af = __shfl_sync(full, acc, f);
            if (ok && lane > f) {
              const double v = ((lm >> f) & 1u)
                                   ? s_y[f][lane] + s_y[lane][f]
                                   : f4_side(cl[cur][f], false, jj, dvr4, rbndsq) +
                                         f4_side(cl[cur][f], true, jj, dvr4, rbndsq);
              part += af ? v : -v;
              acc = !(speak <= (dptmn + dptfc * part) && spp == 0.);
            }
            if (lane == f) live = acc;
            mis = __ballot_sync(full, acc != live) & ~((2u << f) - 1u);
          }
          // the first accepted line at or beyond VNULST ends the window (:3928, IHI=-1)
          const unsigned tm = __ballot_sync(full, acc && vnu >= W.vnulst);
          const int lim = tm ? __ffs(tm) - 1 : kChunk;
          const unsigned am = __ballot_sync(full, acc && has != 0 && lane < lim);
          const int rank = __popc(am & ((1u << lane) - 1u));
          if ((am >> lane) & 1u) s_idx[cur][rank] = lane;
          const unsigned imgp =
              __reduce_or_sync(full, (((am >> lane) & 1u) && (has & 2)) ? (1u << rank) : 0u);
          if (lane == 0) {
            s_nacc[cur] = __popc(am);
            s_imgp[cur] = imgp;
            if (tm) s_stop = 1;
          }
          decided = 1;
        }
        if (lane == 0) s_state[ph & 1] = decided;
      } else if (warp == 1) {
        if (go) build(nxt);
        else if (lane == 0) s_nval[nxt] = 0;
      }
    } else if (have_prev) {
      // adders: chunk t-1's accepted lines over the whole window
      const int ad = (int)threadIdx.x - 32 * DEC;
      const int na = s_nacc[prv];
      if constexpr (sizeof(T) == 8) {
        // FP64: each point summed in shared memory line by line, line
        // before image, in CONVF4's order
#pragma unroll
        for (int q = 0; q < kFwPts; q++) {
          const int j = 1 + ad + kFwAdders * q;
          if (j <= npt) R4w[j] = R4r[j];
        }
        for (int a = 0; a < na; a++) {
          const Line& pl = cl[prv][s_idx[prv][a]];
#pragma unroll 1
          for (int m = 0; m < 2; m++) {
            const int lo = m ? pl.mjmin : pl.jmin, hi = m ? pl.mjmax : pl.jmax;
            // this adder's points j = 1 + ad + kFwAdders q inside [lo, hi]
            const int qlo = (lo - 1 - ad <= 0) ? 0 : (lo - 2 - ad) / kFwAdders + 1;
            const int qhi = (hi - 1 - ad < 0) ? -1 : (hi - 1 - ad) / kFwAdders;
            if (qhi < qlo) continue;
            F4Reg<double> rg;
            f4_load(rg, pl, m, 0);
            // the offset to the line centre advances by kFwAdders points a
            // step (CONVF4 accumulates XJJ the same way); the bound term and
            // the coupling factor are fixed per line
            const double step = double(kFwAdders) * dvr4;
            double xm = double(ad + kFwAdders * qlo) * dvr4 - rg.xnui;
            if (!rg.co2 && rg.dptrat == 0.) {
#pragma unroll 2
              for (int q = qlo; q <= qhi; q++, xm += step) {
                const double xmsq = xm * xm;
                const double zvsq = xmsq * rg.rvi2;
                const double f = zvsq <= 4096. ? (rg.sa3 + zvsq * rg.sb3) - rg.f4bnd
                                               : rg.sil * recip_nr(rg.alfl2 + xmsq) - rg.f4bnd;
                R4w[1 + ad + kFwAdders * q] += f;
              }
            } else {
#pragma unroll 2
              for (int q = qlo; q <= qhi; q++, xm += step) {
                const double xmsq = xm * xm;
                const double zvsq = xmsq * rg.rvi2;
                const double sub = rg.co2 ? (2. - xmsq * rbndsq) * rg.f4bnd : rg.f4bnd;
                double f = zvsq <= 4096. ? (rg.sa3 + zvsq * rg.sb3) - sub
                                         : rg.sil * recip_nr(rg.alfl2 + xmsq) - sub;
                f = f + xm * rg.dptrat * f;
                R4w[1 + ad + kFwAdders * q] += f;
              }
            }
            nevals += (unsigned)(qhi - qlo + 1);
          }
        }
      } else {
        // split precision: the chunk's lines summed in FP32 in shared memory
        // (each adder its own points), the chunk total added to the FP64 R4
        float* acc32 = reinterpret_cast<float*>(fw_r4 + 2 * kR4Stride) + ad;
        const float dvr4f = (float)dvr4, bndf = (float)bnd, rbndsqf = (float)rbndsq;
        for (int a = 0; a < na; a++) {
          const Line& pl = cl[prv][s_idx[prv][a]];
#pragma unroll 1
          for (int m = 0; m < 2; m++) {
            const int lo = m ? pl.mjmin : pl.jmin, hi = m ? pl.mjmax : pl.jmax;
            const int qlo = (lo - 1 - ad <= 0) ? 0 : (lo - 2 - ad) / kFwAdders + 1;
            const int qhi = (hi - 1 - ad < 0) ? -1 : (hi - 1 - ad) / kFwAdders;
            if (qhi < qlo) continue;
            F4Reg<float> rg;
            f4_load(rg, pl, m, 1 + ad);
#pragma unroll 2
            for (int q = qlo; q <= qhi; q++)
              acc32[kFwAdders * q] += f4_at(rg, 0, rg.k0 + (float)(kFwAdders * q), dvr4, rbndsq,
                                            dvr4f, bndf, rbndsqf);
            nevals += (unsigned)(qhi - qlo + 1);
          }
        }
#pragma unroll
        for (int q = 0; q < kFwPts; q++) {
          const int j = 1 + ad + kFwAdders * q;
          if (j <= npt) R4w[j] = R4r[j] + (double)acc32[kFwAdders * q];
          acc32[kFwAdders * q] = 0.f;
        }
      }
    }
    __syncthreads();
    const int decided = s_state[ph & 1];
    if (have_prev) rb ^= 1;
    cur = nxt;
    have_prev = decided != 0;
    if (!decided) break;
  }
  // one counter update per warp
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) nevals += __shfl_xor_sync(0xffffffffu, nevals, o);
  if ((threadIdx.x & 31) == 0 && nevals) atomicAdd(&w.counters[0], nevals);
  double* R4s = fw_r4 + rb * kR4Stride;
  double* out = w.r4 + (int64_t)gw * kR4Stride;
  if (L.jrad == 1) {
    // radiation field applied to R4 (LBLF4 :3726-3758)
    if (threadIdx.x == 0) {
      const double xkt = 1. / L.beta_f;
      double vitst = W.v1r4 - dvr4, rdlast = -1.;
      long n1 = 0, n2 = 0;
      do {
        n1 = n2 + 1;
        double vi = W.v1r4 + dvr4 * double(n1 - 1), rdel;
        double rv = radfni(vi, dvr4, xkt, vitst, rdel, rdlast);
        n2 = fint((vitst - W.v1r4) / dvr4 + 0.001);
        if (n2 > npt) n2 = npt;
        for (long i = n1; i <= n2; i++) {
          R4s[i] = R4s[i] * rv;
          rv = rv + rdel;
        }
      } while (n2 < npt);
    }
    __syncthreads();
  }
  for (int j = threadIdx.x; j < kR4Stride; j += kFwThreads) out[j] = (j >= 1 && j <= npt) ? R4s[j] : 0.;
}

// =========================================================================
// RDLIN/LNCOR1 near-wing line scaling and rejection (src/oprop.f90:678-1197),
// one CTA per layer walking the TAPE3 panels in order: each panel's lines are
// scaled with the far-wing window and panel origin current when HIRAC1 reads
// that panel, which is the first panel able to hold all earlier accepted lines.
// =========================================================================
__device__ __forceinline__ long jmax1_at(double vnu, double vft, double dv, double bhw) {
  return fint((vnu - vft) / dv + bhw + 1.5);
}

// Inclusive max-scan over the CTA's threads in thread order.
__device__ int block_max_scan(int v, int* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v = max(v, t);
  }
  if (lane == 31) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    int t = lane < (int)(blockDim.x >> 5) ? sh[lane] : -1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t = max(t, u);
    }
    sh[lane] = t;
  }
  __syncthreads();
  const int r = (wid > 0) ? max(v, sh[wid - 1]) : v;
  __syncthreads();
  return r;
}

// RDLIN/LNCOR1 per near-wing line and layer, everything that does not
// depend on the TAPE3 panel being read (src/oprop.f90:678-1197): strength
// scaling and rejection, widths, the Voigt interpolation index and the
// CNVFNV sub-function strengths (written to their final slots), the reach
// 64 ALFV + VNU of the VFT cut, the peak SPEAK of the R4 test and the first
// panel able to hold the line's R1 window, all in one NearPre record.
__global__ void __launch_bounds__(256) k_near_lines(Work w, DevLines ln) {
  const int l = blockIdx.y;
  const LayerDev& L = w.L[l];
  const int32_t k = (int32_t)(blockIdx.x * blockDim.x + threadIdx.x);
  const int32_t nn = (int32_t)(L.near_hi - L.near_lo);
  if (k >= nn) return;
  const int32_t i = (int32_t)L.near_lo + k;
  const int64_t slot = (int64_t)k + L.off_near;
  const double DV = L.dv;
  NearPre pre = {0., 0., 0., 0, -1};  // flags 0: rejected
  if (ln.iflg[i] >= 0) {
    const int mcode = ln.mol[i];
    const int m = mcode % 100, iso = (mcode % 1000) / 100;
    double sui = 0.;
    bool rej = !(m >= 1 && m <= 47 && iso >= 1 && iso <= c_isomax[m]);
    if (!rej) {
      const double wkm = (m <= L.nmol) ? L.wk[m] : 0.;
      sui = (double)ln.sp[i] * wkm;
      if (L.jrad == 1) sui = sui * radfn(ln.vnu[i], L.xkt);
      if (sui == 0.) rej = true;
    }
    if (!rej) {
      const int iflag = ln.iflg[i];
      double yi = 0., gi = 0., g1 = 0., g2 = 0.;
      if (iflag == 1 || iflag == 3)
        coupling(ln, i, iflag, L.ilc_n, L.rectlc_n, L.tmpdif_n, false, yi, gi, g1, g2);
      const double vnu = ln.vnu[i] + L.rhorat * (double)ln.pshift[i];
      const double tmpcor = pow(L.tratio, (double)ln.tmpalf[i]);
      const double a0 = air_width(ln, i, m) * tmpcor;
      const double hs = (double)ln.hwhms[i] * tmpcor;
      double alfl = a0 * (L.rhorat - L.rhoslf[m]) + hs * L.rhoslf[m];
      if (iflag == 3) alfl = alfl * (1.0 - g1 * L.pavp0 - g2 * L.pavp2);
      const double alfad = vnu * L.alfd1[m][iso];
      const double zeta = alfl / (alfl + alfad);
      const double fz = 100. * zeta;
      long iz = fint(fz + kONEPL);
      iz = iz < 1 ? 1 : (iz > 101 ? 101 : iz);
      const double zd = fz - double(iz - 1);
      double alfv = (c_avrat[iz - 1] + zd * (c_avrat[iz] - c_avrat[iz - 1])) * (alfl + alfad);
      if (alfv < DV) alfv = DV;
      if (alfv > L.alfmax) alfv = L.alfmax;
      const double reach = 64. * alfv + vnu;  // HWF3*ALFV+VNU (:1120)
      const double recalf = 1. / alfv;
      double epp = (double)ln.epp[i];
      if (epp <= -1.001) epp = fabs(epp);
      if (epp > -0.999)
        sui = sui * L.scor[m][iso] * exp(-epp * L.betacr_n) * (1. + exp(-vnu / L.xkt));
      const double sp = sui * (1. + gi * L.pavp2);
      const double sppsp = (sui * yi * L.pavp0) / sp;
      bool r4test = false;
      double speak = 0.;
      if (iflag == 0) {
        speak = sui * recalf;
        if (L.dvr4 <= 0.) {
          if (speak <= L.dptmn) rej = true;
        } else {
          r4test = (sppsp == 0.);
        }
      }
      if (!rej) {
        // strengths of the sub-functions (CNVFNV :1270-1282)
        const double depth = sp * recalf;
        double* str = w.n_str + 5 * slot;
        const double* cf[5] = {c_cf1, c_cf2, c_cf3, c_cgauss, c_cer};
#pragma unroll
        for (int q = 0; q < 5; q++) str[q] = depth * (cf[q][iz - 1] + zd * (cf[q][iz] - cf[q][iz - 1]));
        w.n_sppsp[slot] = sppsp;
        const double zslope = recalf * L.wavdxf;
        const double bhw = kHWDXF / zslope;
        // First panel whose buffer holds the line's R1 window (JMAX1 <=
        // MAX1).  JMAX1 falls as the panel origin rises, so the panel the
        // reference settles on from read panel P is the later of P and this.
        const double* vft = w.vft + L.off_panel;
        const int npanel = (int)L.npanel;
        int p = 0;
        const long excess = jmax1_at(vnu, vft[0], DV, bhw) - L.max1;
        if (excess > 0) p = (int)min((excess + 2399) / 2400, (long)npanel);
        while (p > 0 && jmax1_at(vnu, vft[p - 1], DV, bhw) <= L.max1) p--;
        while (p < npanel && jmax1_at(vnu, vft[p], DV, bhw) > L.max1) p++;
        w.n_zslope[slot] = zslope;
        // the R4 point of the R4 test in the window of that panel, which
        // is the read panel's window for most lines
        int32_t wj = -1;  // none
        if (r4test && L.nwin > 0 && L.nwin < 32768) {
          const int wq = w.win_of[L.off_panel + (p < npanel ? p : npanel - 1)];
          const WinDev& W = w.win[L.off_win + wq];
          long jj = fint((vnu - W.v1r4) / L.dvr4 + 1.);
          jj = jj < 1 ? 1 : (jj > W.nptr4 ? W.nptr4 : jj);
          wj = (int32_t)((wq << 16) | (int)jj);
        }
        pre = {vnu, reach, speak, (p << 2) | 1 | (r4test ? 2 : 0), wj};
      }
    }
  }
  w.n_pre[slot] = pre;
}

// LNCOR1's tests that depend on the TAPE3 panel being read: the VFT cut
// (:1120) and, for uncoupled lines, the R4 rejection against the window of
// the read panel (:1160-1175).  r4 is that window's R4.
__device__ __forceinline__ bool near_accept(const NearPre& r, double vft_read, int wi,
                                            double v1r4, int nptr4, const double* r4,
                                            double dvr4, double dptmn, double dptfc) {
  bool ok = (r.pf_fl & 1) && !(r.reach < vft_read);
  if (ok && (r.pf_fl & 2) && wi >= 0) {
    long jj;
    if ((r.wj >> 16) == wi) {
      jj = r.wj & 0xffff;  // computed for this window by k_near_lines
    } else {
      jj = fint((r.vnu - v1r4) / dvr4 + 1.);
      jj = jj < 1 ? 1 : (jj > nptr4 ? nptr4 : jj);
    }
    if (r.speak <= (dptmn + dptfc * r4[jj])) ok = false;
  }
  return ok;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// The read-panel walk of LNCOR1, one warp per layer over its TAPE3 panels
// in order.  The panel read next is the first panel able to hold the R1
// windows of all lines accepted so far (JMAX1 <= MAX1); a line that no
// panel can hold ends the walk (CNVFNV never reaches it or what follows).
// Per TAPE3 panel the walk records the read panel and the first line not
// reached; k_near_out derives everything else in parallel.  Line records
// arrive in shared memory kWalkRing-1 panels ahead by asynchronous copies.
__global__ void __launch_bounds__(32) k_near_walk(Work w, DevLines ln) {
  extern __shared__ double sm[];
  const int l = blockIdx.x;
  const int lane = threadIdx.x;
  const unsigned full = 0xffffffffu;
  const LayerDev& L = w.L[l];
  const int npanel = (int)L.npanel, nwin = (int)L.nwin;
  const int64_t blk_lo = L.blk_lo, nblk = L.blk_hi - L.blk_lo;
  const int64_t near_lo = L.near_lo, near_hi = L.near_hi, off_near = L.off_near;
  const int64_t off_win = L.off_win, off_nblk = L.off_nblk;
  const double dvr4 = L.dvr4, dptmn = L.dptmn, dptfc = L.dptfc;
  double* s_r4 = sm;  // first: 16-byte aligned for the asynchronous copies
  double* s_vft = s_r4 + kR4Stride;
  double* s_v1r4 = s_vft + npanel;
  const size_t dbytes = ((size_t)(npanel + nwin + kR4Stride) * sizeof(double) + 31) / 32 * 32;
  NearPre* ring = reinterpret_cast<NearPre*>(reinterpret_cast<char*>(sm) + dbytes);
  int32_t* s_wof = reinterpret_cast<int32_t*>(ring + kWalkRing * 256);
  int32_t* s_nptr4 = s_wof + npanel;
  constexpr int kBs = 64;
  __shared__ int64_t s_bs[kBs + 1];
  __shared__ int32_t s_rn[kWalkRing];
  for (int k = lane; k < npanel; k += 32) {
    s_vft[k] = w.vft[L.off_panel + k];
    s_wof[k] = nwin > 0 ? w.win_of[L.off_panel + k] : -1;
  }
  for (int k = lane; k < nwin; k += 32) {
    s_v1r4[k] = w.win[off_win + k].v1r4;
    s_nptr4[k] = w.win[off_win + k].nptr4;
  }
  // TAPE3 panel starts of panels [bs_base, bs_base + kBs]
  int64_t bs_base = -(int64_t)kBs - 2;
  // copy the records of near-range panel bi into ring slot bi % kWalkRing
  auto issue = [&](int64_t bi) {
    if (bi < nblk) {
      const int64_t b = blk_lo + bi;
      if (b + 1 > bs_base + kBs) {
        __syncwarp();
        for (int k = lane; k <= kBs; k += 32) s_bs[k] = (b + k <= L.blk_hi) ? ln.bs[b + k] : 0;
        bs_base = b;
        __syncwarp();
      }
      const int64_t a = s_bs[b - bs_base] > near_lo ? s_bs[b - bs_base] : near_lo;
      const int64_t e = s_bs[b + 1 - bs_base] < near_hi ? s_bs[b + 1 - bs_base] : near_hi;
      const int n = e > a ? (int)(e - a) : 0;  // at most 250 (RDLIN's LIMIN)
      NearPre* dst = ring + (bi % kWalkRing) * 256;
      const NearPre* src = w.n_pre + off_near + (a - near_lo);
      for (int k = lane; k < n; k += 32) {
        cp_async16(dst + k, src + k);
        cp_async16(reinterpret_cast<char*>(dst + k) + 16, reinterpret_cast<const char*>(src + k) + 16);
      }
      if (lane == 0) s_rn[bi % kWalkRing] = n;
    }
    cp_async_commit();
  };
  __syncwarp();
  for (int64_t bi = 0; bi < kWalkRing - 1; bi++) issue(bi);
  int pread = 0, rwin = -1;
  int packed = 0;  // accepted lines of the panels walked so far
  bool stopped = false;
  for (int64_t bi = 0; bi < nblk; bi++) {
    issue(bi + kWalkRing - 1);
    cp_async_wait<kWalkRing - 1>();
    __syncwarp();
    const int slot = (int)(bi % kWalkRing);
    const int n = s_rn[slot];
    const NearPre* rb = ring + slot * 256;
    int stop = INT_MAX;
    if (!stopped) {
      const double vft_read = s_vft[pread];
      const int wi = nwin > 0 ? s_wof[pread] : -1;
      if (wi >= 0 && wi != rwin && dvr4 > 0.) {
        // the window's R4 (kR4Stride doubles, a multiple of 16 bytes)
        const double* r4 = w.r4 + (off_win + wi) * kR4Stride;
        for (int k = 2 * lane; k < (int)kR4Stride; k += 64) cp_async16(s_r4 + k, r4 + k);
        cp_async_commit();
        cp_async_wait<0>();
        rwin = wi;
        __syncwarp();
      }
      const double v1r4 = wi >= 0 ? s_v1r4[wi] : 0.;
      const int nptr4 = wi >= 0 ? s_nptr4[wi] : 0;
      int pf[8];
      int first_out = INT_MAX;  // this lane's first accepted line no panel holds
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int k = lane + 32 * j;
        pf[j] = -1;
        if (k < n) {
          const NearPre r = rb[k];
          if (near_accept(r, vft_read, wi, v1r4, nptr4, s_r4, dvr4, dptmn, dptfc)) {
            pf[j] = max(pread, r.pf_fl >> 2);
            if (pf[j] >= npanel && k < first_out) first_out = k;
          }
        }
      }
      stop = __reduce_min_sync(full, first_out);
      int pm = pread;
#pragma unroll
      for (int j = 0; j < 8; j++)
        if (lane + 32 * j < stop) pm = max(pm, pf[j]);
      const int pmax = __reduce_max_sync(full, pm);
      // accepted lines of this panel that CNVFNV reaches: their ranks in the
      // layer's packed list start at `packed`
      int cnt = 0;
#pragma unroll
      for (int j = 0; j < 8; j++)
        if (pf[j] >= 0 && lane + 32 * j < stop) cnt++;
      cnt = __reduce_add_sync(full, cnt);
      if (lane == 0) {
        w.n_blk[off_nblk + bi] = make_int2(pread, stop);
        w.n_boff[off_nblk + bi] = packed;
      }
      packed += cnt;
      pread = pmax;
      if (stop != INT_MAX) stopped = true;
    } else if (lane == 0) {
      w.n_blk[off_nblk + bi] = make_int2(-1, 0);
      w.n_boff[off_nblk + bi] = packed;
    }
    __syncwarp();  // the slot is refilled by the next issue
  }
  cp_async_wait<0>();
  if (lane == 0) {
    w.n_cnt[l] = packed;
    w.n_hw3[l] = 0;
  }
}

// Window limits of every near-wing line (one CTA per layer and TAPE3
// panel), from the read panel and stop line the walk recorded: the line is
// accepted by the same tests, and CNVFNV convolves it in the panel current
// when it reaches it: the read panel or later, as far as the earlier lines
// of the panel pushed it (:1283-1305).
__global__ void __launch_bounds__(256) k_near_out(Work w, DevLines ln) {
  __shared__ int s_scan[32];
  const int l = blockIdx.y;
  const LayerDev& L = w.L[l];
  const int64_t bi = blockIdx.x;
  if (bi >= L.blk_hi - L.blk_lo) return;
  const int64_t b = L.blk_lo + bi;
  const int tid = threadIdx.x;
  const int64_t a = ln.bs[b] > L.near_lo ? ln.bs[b] : L.near_lo;
  const int64_t e = ln.bs[b + 1] < L.near_hi ? ln.bs[b + 1] : L.near_hi;
  const int64_t i = a + tid;
  const bool in = i < e;
  const int64_t slot = (i - L.near_lo) + L.off_near;
  const int2 pb = w.n_blk[L.off_nblk + bi];
  const int pread = pb.x;
  bool ok = false;
  int pfit = -1;
  NearPre r;
  if (in && pread >= 0) {
    r = w.n_pre[slot];
    const int64_t pp = L.off_panel + pread;
    const int wi = L.nwin > 0 ? w.win_of[pp] : -1;
    double v1r4 = 0.;
    int nptr4 = 0;
    const double* r4 = w.r4;
    if (wi >= 0) {
      v1r4 = w.win[L.off_win + wi].v1r4;
      nptr4 = w.win[L.off_win + wi].nptr4;
      r4 = w.r4 + (L.off_win + wi) * kR4Stride;
    }
    ok = near_accept(r, w.vft[pp], wi, v1r4, nptr4, r4, L.dvr4, L.dptmn, L.dptfc) && tid < pb.y;
    if (ok) pfit = max(pread, r.pf_fl >> 2);
  }
  const int pconv = max(pread, block_max_scan(ok ? pfit : -1, s_scan));
  // rank in the layer's packed list: the panel's start (from the walk) plus
  // the accepted lines before this one in the panel
  __shared__ int s_wc[8];
  const int lane = tid & 31, warp = tid >> 5;
  const unsigned m = __ballot_sync(0xffffffffu, ok);
  if (lane == 0) s_wc[warp] = __popc(m);
  __syncthreads();
  unsigned ntrip = 0;
  int hw = 0;
  if (ok) {
    int rank = w.n_boff[L.off_nblk + bi] + __popc(m & ((1u << lane) - 1u));
    for (int k = 0; k < warp; k++) rank += s_wc[k];
    const double DV = L.dv;
    const double zslope = w.n_zslope[slot];
    const double bhw = kHWDXF / zslope;
    const double zint = (r.vnu - w.vft[L.off_panel + pconv]) / DV;
    const long jmax1 = fint(zint + bhw + 1.5);
    const long jmin1 = fint(zint - bhw + 1.5);
    const double rs = zint < 0.0 ? -0.5 : 0.5;
    const long j2 = fint(zint * (1. - L.conf2) + rs);
    const long j3 = fint(zint * (1. - L.conf3) + rs);
    ntrip = (unsigned)(jmax1 - jmin1 + 1);
    // the record: CNVFNV's constants and the windows on the three global
    // grids (the convolution panel's windows shifted by 2400/600/150 points
    // per panel)
    const double* sv = w.n_str + 5 * slot;
    NearRec q;
    q.zint = zint;
    q.zslope = zslope;
    q.sppsp = w.n_sppsp[slot];
    q.s0 = sv[0];
    q.s2 = sv[1];
    q.s3 = sv[2];
    q.sg = sv[3];
    q.sx = sv[4];
    q.lo1 = (int32_t)jmin1 + 2400 * pconv;
    q.hi1 = (int32_t)jmax1 + 2400 * pconv;
    q.lo2 = (int32_t)(jmin1 - j2) + 600 * pconv;
    q.hi2 = (int32_t)(jmax1 - j2) + 600 * pconv;
    q.lo3 = (int32_t)(jmin1 - j3) + 150 * pconv;
    q.hi3 = (int32_t)(jmax1 - j3) + 150 * pconv;
    q.pc = pconv;
    q.pad = 0;
    w.n_rec[L.off_near + rank] = q;
    const double v = ln.vnu[i];
    w.n_rvnu[L.off_near + rank] = v;
    // R3 half-window about the TAPE3 centre (g at VFT0 + (g-1) DVR3)
    const double c3 = (v - L.vft0) / L.dvr3 + 1.;
    hw = (int)ceil(fmax(c3 - double(q.lo3), double(q.hi3) - c3));
  }
  // one update per warp of the near point-triple counter (a single address
  // updated by every line would serialise the kernel) and of the layer's
  // widest R3 half-window
  const unsigned wsum = __reduce_add_sync(0xffffffffu, ntrip);
  if (lane == 0 && wsum) atomicAdd(&w.counters[1], (unsigned long long)wsum);
  const int whw = __reduce_max_sync(0xffffffffu, hw);
  if (lane == 0 && m) atomicMax(&w.n_hw3[l], whw);
}

__device__ int64_t lower_bound_d(const double* v, int64_t lo, int64_t hi, double x) {
  while (lo < hi) {
    int64_t m = (lo + hi) >> 1;
    if (v[m] < x) lo = m + 1;
    else hi = m;
  }
  return lo;
}

// =========================================================================
// Continuum: mt_ckd_h2o_absco + CONTNM (mt_ckd_h2o_module.f90:68-174,
// contnm.f90:279-311), one CTA per layer onto the 1 cm-1 ABSRB grid.
// =========================================================================
// The H2O self and foreign part of CONTNM (mt_ckd_h2o_absco onto the 1 cm-1
// grid, src/contnm.f90:199-324), assigned to ABSRB.
__device__ void h2o_part(const LayerDev& L, const DevMtckd& ck, double h2o_fac, double* absrb,
                         double xself, double xfrgn) {
  const double wv1 = L.v1abs, wv2 = L.v2abs, dva = L.dvabs;
  auto wvn = [&](int64_t i) { return ck.v0 + ck.dv * double(i - 1); };
  __shared__ int64_t s_i1, s_i2;
  if (threadIdx.x == 0) {
    const double dvc = wvn(2) - wvn(1);
    int64_t i = 1;
    while (i < ck.n && wvn(i) <= (wv1 - 2 * dvc)) i++;
    int64_t i1 = i - 1;
    if (i1 == 0) i1 = 1;
    while (i < ck.n && wvn(i) < (wv2 + 2 * dvc)) i++;
    s_i1 = i1;
    s_i2 = i;
  }
  __syncthreads();
  const int64_t i1 = s_i1, i2 = s_i2;
  const int64_t ncoeff = i2 - i1 + 1;
  const double xkt = L.tave / kRADCN2;
  const double rho = (L.pave / ck.ref_press) * (ck.ref_temp / L.tave);
  const bool radflag = (L.jrad != 0);
  const double dvc = wvn(2) - wvn(1);
  const int64_t nptabs = fint((wv2 - wv1) / dva + 1);
  int64_t ist = fint(2 + (wvn(1) - wv1) / dva + 1.e-5);
  if (ist < 1) ist = 1;
  int64_t lst = fint(1 + (wvn(ck.n) - wv1) / dva + 1.e-5);
  if (lst > nptabs) lst = nptabs;
  const double v1a = wvn(i1), v2a = wvn(i2);
  int64_t ilo = fint((v1a + dvc - wv1) / dva + 1. + kONEMI);
  if (ilo < ist) ilo = ist;
  int64_t ihi = fint((v2a - dvc - wv1) / dva + kONEMI);
  if (ihi > lst) ihi = lst;
  auto coef = [&](int64_t k, bool self) -> double {
    if (k < 1 || k > ncoeff) return 0.;
    const int64_t ii = i1 + k - 1;
    const double vi = wvn(ii);
    double c;
    if (self)
      c = ck.self[ii - 1] * pow(ck.ref_temp / L.tave, ck.texp[ii - 1]) * h2o_fac * rho;
    else
      c = ck.forn[ii - 1] * (1 - h2o_fac) * rho;
    if (radflag) {
      const double x = vi / xkt;
      double r = vi;
      if (x <= 0.01) r = 0.5 * x * vi;
      else if (x <= 10.) {
        const double e = exp(-x);
        r = vi * (1 - e) / (1. + e);
      }
      c = c * r;
    }
    return c;
  };
  const double rec = 1. / dvc;
  for (int64_t I = ilo + threadIdx.x; I <= ihi; I += blockDim.x) {
    const double vi = wv1 + dva * double(I - 1);
    const long J = fint((vi - v1a) * rec + kONEPL);
    const double vj = v1a + dvc * double(J - 1);
    const double p = rec * (vi - vj);
    const double C = (3. - 2. * p) * p * p;
    const double B = 0.5 * p * (1. - p);
    const double b1 = B * (1. - p), b2 = B * p;
    double cs = -coef(J - 1, true) * b1 + coef(J, true) * (1. - C + b2) +
                coef(J + 1, true) * (C + b1) - coef(J + 2, true) * b2;
    double cf = -coef(J - 1, false) * b1 + coef(J, false) * (1. - C + b2) +
                coef(J + 1, false) * (C + b1) - coef(J + 2, false) * b2;
    absrb[I] = L.wk[1] * cs * xself + L.wk[1] * cf * xfrgn;
  }
}

// The continua of CONTNM after H2O (src/contnm.f90:326-994) each tabulate
// coefficients on a coarse grid of their own (V1S, DVS, NPTS), set up alike
// (FRNCO2 :1322-1337 and its siblings): from one point below V1ABS-DVS to
// one above V2ABS+DVS.  The layer's coefficients C(J) on that grid are
// added to ABSRB by XINT between pre_xint's IST and LAST (:994-1012); the
// four C(J) a point's interpolation needs are formed where used.
struct CoarseGrid {
  int64_t i1, nptc;
  double v1c, v2c, dvc;
};
__device__ CoarseGrid coarse_grid(double V1S, double DVS, int64_t NPTS, const LayerDev& L) {
  CoarseGrid g;
  g.dvc = DVS;
  const double v1c = L.v1abs - DVS, v2c = L.v2abs + DVS;
  g.i1 = (v1c < V1S) ? -1 : fint((v1c - V1S) / DVS + 0.01);
  g.v1c = V1S + DVS * double(g.i1 - 1);
  const int64_t i2 = fint((v2c - V1S) / DVS + 0.01);
  g.nptc = i2 - g.i1 + 3;
  if (g.nptc > NPTS) g.nptc = NPTS + 4;
  g.v2c = g.v1c + DVS * double(g.nptc - 1);
  return g;
}

// XINT (src/oprop.f90:2201-2234, AFACT = 1) of C(J) = coef(J, VJ) (0 for J
// outside 1..NPTC) onto the layer's ABSRB points, the block's threads
// taking points in turn.
template <typename Coef>
__device__ void xint_coarse(const LayerDev& L, const CoarseGrid& g, double V1SS, double V2SS,
                            Coef coef, double* absrb) {
  auto C = [&](int64_t j) -> double {
    return (j < 1 || j > g.nptc) ? 0. : coef(j, g.v1c + g.dvc * double(j - 1));
  };
  int64_t ist = fint(2 + (V1SS - L.v1abs) / L.dvabs + 1.e-5);
  if (ist < 1) ist = 1;
  int64_t last = fint(1 + (V2SS - L.v1abs) / L.dvabs + 1.e-5);
  if (last > L.nptabs) last = L.nptabs;
  const double rec = 1. / g.dvc;
  int64_t ilo = fint((g.v1c + g.dvc - L.v1abs) / L.dvabs + 1. + kONEMI);
  if (ilo < ist) ilo = ist;
  int64_t ihi = fint((g.v2c - g.dvc - L.v1abs) / L.dvabs + kONEMI);
  if (ihi > last) ihi = last;
  for (int64_t I = ilo + threadIdx.x; I <= ihi; I += blockDim.x) {
    const double vi = L.v1abs + L.dvabs * double(I - 1);
    const int64_t J = fint((vi - g.v1c) * rec + kONEPL);
    const double vj = g.v1c + g.dvc * double(J - 1);
    const double p = rec * (vi - vj);
    const double Cq = (3. - 2. * p) * p * p;
    const double B = 0.5 * p * (1. - p);
    const double b1 = B * (1. - p), b2 = B * p;
    const double conti =
        -C(J - 1) * b1 + C(J) * (1. - Cq + b2) + C(J + 1) * (Cq + b1) - C(J + 2) * b2;
    absrb[I] = absrb[I] + conti * 1.0;
  }
}

__device__ const double d_fco2[LBL_FCO2_N] = {LBL_FCO2_VALUES};
__device__ const double d_xfacco2[500] = {LBL_XFACCO2_VALUES};
__device__ const double d_co2_tdep[25] = {LBL_CO2_TDEP_VALUES};
__device__ const double d_o2f_x[LBL_O2F_N] = {LBL_O2F_XO2_VALUES};
__device__ const double d_o2f_t[LBL_O2F_N] = {LBL_O2F_XO2T_VALUES};
__device__ const double d_n2r_c296[LBL_N2R296_N] = {LBL_N2R296_C_VALUES};
__device__ const double d_n2r_sf296[LBL_N2R296_N] = {LBL_N2R296_SF_VALUES};
__device__ const double d_n2r_c220[LBL_N2R220_N] = {LBL_N2R220_C_VALUES};
__device__ const double d_n2r_sf220[LBL_N2R220_N] = {LBL_N2R220_SF_VALUES};
__device__ const double d_n2f_272[LBL_N2F_N] = {LBL_N2F_X272_VALUES};
__device__ const double d_n2f_228[LBL_N2F_N] = {LBL_N2F_X228_VALUES};
__device__ const double d_n2f_ah2o[LBL_N2F_N] = {LBL_N2F_AH2O_VALUES};
__device__ const double d_n2o1[LBL_N2O1_N] = {LBL_N2O1_X_VALUES};
__device__ const double d_o2i1[LBL_O2I1_N] = {LBL_O2I1_X_VALUES};

struct ContScale {
  double xco2c, xo2cn, xn2cn;
};

// CO2 (:326-378, FRNCO2 :1295-1349: the band-head temperature dependence
// of points 1196-1220), the mt_ckd_2.5 factors XFACCO2 from 2000 to 2998
// cm-1, WCO2; the O2 collision-induced fundamental (:491-540, o2_ver_1
// :7254-7318); the N2 collision-induced rotational band (:745-792, xn2_r
// :2497-2566) and fundamental (:811-858, n2_ver_1 :2668-2754); each times
// the radiation term on its coarse grid when JRAD=1, and added in CONTNM's
// order.
__device__ void cia_parts(const LayerDev& L, const ContScale& xs, double* absrb) {
  const double xkt = L.tave / kRADCN2;
  const double rhoave = (L.pave / 1013.) * (296. / L.tave);
  const double amagat = (L.pave / 1013.) * (273. / L.tave);
  const double x_h2o = L.wk[1] / L.wtot, x_o2 = L.wk[7] / L.wtot;
  const double x_n2 = 1. - x_h2o - x_o2;
  const double wn2 = x_n2 * L.wtot;
  const double xlosmt = 2.68675E+19;
  auto rad = [&](double c, double vj) { return L.jrad == 1 ? c * radfn(vj, xkt) : c; };
  if ((L.v2 > -20.0) && (L.v1 < 10000.) && xs.xco2c > 0.) {
    __syncthreads();
    const double wco2 = L.wk[2] * rhoave * 1.0E-20 * xs.xco2c;
    const double trat = L.tave / LBL_CO2_TEFF;
    const CoarseGrid g = coarse_grid(LBL_FCO2_V1, LBL_FCO2_DV, LBL_FCO2_N, L);
    xint_coarse(L, g, LBL_FCO2_V1, LBL_FCO2_V2, [&](int64_t j, double vj) {
      const int64_t I = g.i1 + (j - 1);
      double c = 0.;
      if (I >= 1 && I <= LBL_FCO2_N) {
        double tcor = 1.;
        if (I >= 1196 && I <= 1220) tcor = pow(trat, d_co2_tdep[I - 1196]);
        c = tcor * d_fco2[I - 1];
      }
      double cfac = 1.;
      if (vj >= 2000. && vj <= 2998.) cfac = d_xfacco2[fint((vj - 1998.) / 2. + 0.00001) - 1];
      c = cfac * c;
      return rad(c * wco2, vj);
    }, absrb);
  }
  if ((L.v2 > 1340.0) && (L.v1 < 1850.) && xs.xo2cn > 0.) {
    __syncthreads();
    const double tau_fac = xs.xo2cn * L.wk[7] * 1.e-20 * amagat;
    const double xktfac = (1. / 296.) - (1. / L.tave);
    const double factor = (1.e+20 / xlosmt);
    const CoarseGrid g = coarse_grid(LBL_O2F_V1, LBL_O2F_DV, LBL_O2F_N, L);
    xint_coarse(L, g, LBL_O2F_V1, LBL_O2F_V2, [&](int64_t j, double vj) {
      const int64_t I = g.i1 + (j - 1);
      double c0 = 0.;
      if (I >= 1 && I <= LBL_O2F_N) c0 = factor * d_o2f_x[I - 1] * exp(d_o2f_t[I - 1] * xktfac) / vj;
      return rad(tau_fac * c0, vj);
    }, absrb);
  }
  if ((L.v2 > 7536.0) && (L.v1 < 8500.) && xs.xo2cn > 0.) {
    // the O2 1.27 um band (:543-584, O2INF1 :7384-7440)
    __syncthreads();
    const double tau_fac = xs.xo2cn * (L.wk[7] / xlosmt) * amagat *
                           ((1. / 0.446) * x_o2 + (0.3 / 0.446) * x_n2 + 1. * x_h2o);
    const CoarseGrid g = coarse_grid(LBL_O2I1_V1, LBL_O2I1_DV, LBL_O2I1_N, L);
    xint_coarse(L, g, LBL_O2I1_V1, LBL_O2I1_V2, [&](int64_t j, double vj) {
      const int64_t I = g.i1 + (j - 1);
      const double c0 = (I >= 1 && I <= LBL_O2I1_N) ? d_o2i1[I - 1] / vj : 0.;
      return rad(tau_fac * c0, vj);
    }, absrb);
  }
  if ((L.v2 > -10.0) && (L.v1 < 350.) && xs.xn2cn > 0.) {
    __syncthreads();
    const double tau_fac = xs.xn2cn * (wn2 / xlosmt) * amagat;
    const double tfac = (L.tave - 296.) / (220. - 296.);
    const CoarseGrid g = coarse_grid(LBL_N2R296_V1, LBL_N2R296_DV, LBL_N2R296_N, L);
    xint_coarse(L, g, LBL_N2R296_V1, LBL_N2R296_V2, [&](int64_t j, double vj) {
      const int64_t I = g.i1 + (j - 1);
      double c0 = 0., fo2 = 0.;
      if (I >= 1 && I <= LBL_N2R296_N) {
        c0 = d_n2r_c296[I - 1] * pow(d_n2r_c220[I - 1] / d_n2r_c296[I - 1], tfac);
        const double sf_t = d_n2r_sf296[I - 1] * pow(d_n2r_sf220[I - 1] / d_n2r_sf296[I - 1], tfac);
        fo2 = (sf_t - 1.) * (0.79) / (0.21);
      }
      return rad(tau_fac * c0 * (x_n2 + fo2 * x_o2 + 1. * x_h2o), vj);
    }, absrb);
  }
  if ((L.v2 > 2001.77) && (L.v1 < 2897.59) && xs.xn2cn > 0.) {
    __syncthreads();
    const double tau_fac = xs.xn2cn * (wn2 / xlosmt) * amagat;
    const double T = L.tave;
    const double xtfac = ((1. / T) - (1. / 272.)) / ((1. / 228.) - (1. / 272.));
    const double xt_lin = (T - 272.) / (228. - 272.);
    const double a_o2 = 1.294 - 0.4545 * T / 296.;
    const CoarseGrid g = coarse_grid(LBL_N2F_V1, LBL_N2F_DV, LBL_N2F_N, L);
    xint_coarse(L, g, LBL_N2F_V1, LBL_N2F_V2, [&](int64_t j, double vj) {
      const int64_t I = g.i1 + (j - 1);
      double c0 = 0., c1 = 0., c2 = 0.;
      if (I >= 1 && I <= LBL_N2F_N) {
        const double a = d_n2f_272[I - 1], b = d_n2f_228[I - 1];
        c0 = (a > 0. && b > 0.) ? a * pow(b / a, xtfac) : a + (b - a) * xt_lin;
        c0 = c0 / vj;
        c1 = a_o2 * c0;
        c2 = (9. / 7.) * d_n2f_ah2o[I - 1] * c0;
      }
      return rad(tau_fac * (x_n2 * c0 + x_o2 * c1 + x_h2o * c2), vj);
    }, absrb);
  }
  if ((L.v2 > 4340.0) && (L.v1 < 4910.) && xs.xn2cn > 0.) {
    // the N2 first overtone (:860-906, n2_overtone1 :2916-2968)
    __syncthreads();
    const double tau_fac = xs.xn2cn * (wn2 / xlosmt) * amagat * (x_n2 + 1. * x_o2 + 1. * x_h2o);
    const CoarseGrid g = coarse_grid(LBL_N2O1_V1, LBL_N2O1_DV, LBL_N2O1_N, L);
    xint_coarse(L, g, LBL_N2O1_V1, LBL_N2O1_V2, [&](int64_t j, double vj) {
      const int64_t I = g.i1 + (j - 1);
      const double c0 = (I >= 1 && I <= LBL_N2O1_N) ? d_n2o1[I - 1] / vj : 0.;
      return rad(tau_fac * c0, vj);
    }, absrb);
  }
}

__global__ void k_continuum(Work w, DevMtckd ck, double xself, double xfrgn, double xrayl,
                            ContScale xs) {
  const int l = blockIdx.x;
  const LayerDev& L = w.L[l];
  double* absrb = w.absrb + L.off_abs;  // 1-based, nptabs+4
  for (int64_t j = threadIdx.x; j < L.nptabs + 8; j += blockDim.x) absrb[j] = 0.;
  if (!L.icntnm) return;
  __syncthreads();
  const double h2o_fac = L.h2o_fac;  // WK(1)/WTOT of CONTNM (contnm.f90:261)
  if ((L.v2 > -20.0) && (L.v1 < 20000.) && ((xself > 0.) || (xfrgn > 0)))
    h2o_part(L, ck, h2o_fac, absrb, xself, xfrgn);
  cia_parts(L, xs, absrb);
  // Rayleigh extinction (src/contnm.f90:955-976; no aerosols, IAERSL=0),
  // added to every point of the 1 cm-1 grid after the other parts
  if (L.v2 >= 820. && xrayl > 0.) {
    __syncthreads();
    const double conv_cm2mol = xrayl * 1.E-20 / (2.68675e-1 * 1.e5);
    const double xkt = L.tave / kRADCN2;
    // NPTABS of OPDPTH (src/lblrtm.f90:6222)
    for (int64_t i = 1 + threadIdx.x; i <= L.nptabs; i += blockDim.x) {
      const double vr = L.v1abs + double(i - 1) * L.dvabs;
      const double xv = vr / 1.e4;
      double ray = __dmul_rn(__ddiv_rn(__dmul_rn(__dmul_rn(xv, xv), xv),
                                       __dsub_rn(9.38076E2, __dmul_rn(10.8426, __dmul_rn(xv, xv)))),
                             __dmul_rn(L.wtot, conv_cm2mol));
      if (L.jrad == 1) ray = __dmul_rn(ray, xv);
      else if (L.jrad == 0) ray = __ddiv_rn(__dmul_rn(ray, xv), radfn(vr, xkt));
      absrb[i] += ray;
    }
  }
}

// =========================================================================
// PANEL combination (src/oprop.f90:1371-1561) on the global grids:
//   R3 += XINT(R4 of the panel's window) + XINT(ABSRB)      (:515-519)
//   R2 += 4-point interpolation of R3                        (:1459-1480)
//   OD  = R1 + 4-point interpolation of R2, times RADFNI     (:1482-1519)
// =========================================================================
__device__ __forceinline__ double xint_at(double v1a, double v2a, double dva, const double* A,
                                          double vft, double dvr3, long I, long n1, long n2) {
  const double rec = 1. / dva;
  long ilo = fint((v1a + dva - vft) / dvr3 + 1. + kONEMI);
  if (ilo < n1) ilo = n1;
  long ihi = fint((v2a - dva - vft) / dvr3 + kONEMI);
  if (ihi > n2) ihi = n2;
  if (I < ilo || I > ihi) return 0.;
  const double vi = vft + dvr3 * double(I - 1);
  const long J = fint((vi - v1a) * rec + kONEPL);
  const double vj = v1a + dva * double(J - 1);
  const double p = rec * (vi - vj);
  const double C = (3. - 2. * p) * p * p;
  const double B = 0.5 * p * (1. - p);
  const double b1 = B * (1. - p), b2 = B * p;
  return -A[J - 1] * b1 + A[J] * (1. - C + b2) + A[J + 1] * (C + b1) - A[J + 2] * b2;
}

constexpr double X00 = -7. / 128., X01 = 105. / 128., X02 = 35. / 128., X03 = -5. / 128.,
                 X10 = -1. / 16., X11 = 9. / 16.;

__device__ __forceinline__ double interp4(const double* R, int64_t J, int r) {
  // value added at fine point J*4-3+r from coarse points J-1..J+2; the forms
  // are evaluated and one selected, so neighbouring lanes (with different r)
  // do not diverge; r = 1 and r = 3 are the same weights on the four points
  // taken in opposite order
  const double a = R[J - 1], b = R[J], c = R[J + 1], d = R[J + 2];
  const bool rev = r == 3;
  const double p0 = rev ? d : a, p1 = rev ? c : b, p2 = rev ? b : c, p3 = rev ? a : d;
  const double v13 = X00 * p0 + X01 * p1 + X02 * p2 + X03 * p3;
  const double v2 = X10 * (a + d) + X11 * (b + c);
  return r == 0 ? b : (r == 2 ? v2 : v13);
}

// Global grid index ranges of one panel (panel p of layer L):
//   R1 points whose OD the panel writes, the R2 points their 4-point
//   interpolation reads, and the R3 points those R2 points read.
// Grid indices of a layer fit in 32 bits (a layer holds fewer than 2^31
// points, checked on the host); the panel kernels use 32-bit arithmetic.
struct PanelRange {
  int32_t a1, b1, a2, b2, a3, b3;
  int32_t nhi;
};

__device__ __forceinline__ PanelRange panel_range(const LayerDev& L, int32_t p) {
  PanelRange r;
  const int32_t npanel = (int32_t)L.npanel, n_r2 = (int32_t)L.n_r2, n_r3 = (int32_t)L.n_r3;
  r.nhi = (p == npanel - 1) ? (int32_t)(L.npts - 2400 * (L.npanel - 1) + 32) : 2432;
  r.a1 = 2400 * p + 33;
  r.b1 = 2400 * p + r.nhi;
  r.a2 = (r.a1 - 1) / 4;          // J2 - 1 of the first point
  r.b2 = (r.b1 - 1) / 4 + 3;      // J2 + 2 of the last point
  if (r.b2 > n_r2) r.b2 = n_r2;
  // R2 points that receive R3 are 5 .. n_r2-3 (PANEL :1459-1480)
  const int32_t c2 = r.a2 < 5 ? 5 : r.a2;
  const int32_t d2 = r.b2 > n_r2 - 3 ? n_r2 - 3 : r.b2;
  r.a3 = (c2 - 1) / 4;
  if (r.a3 < 1) r.a3 = 1;
  r.b3 = (d2 - 1) / 4 + 3;
  if (r.b3 > n_r3) r.b3 = n_r3;
  // a first panel starting at or below zero wavenumber folds its grids from
  // point 0 up (RSYM), so it sums them from there
  if (p == 0 && L.vft0 <= 0.) r.a1 = r.a2 = r.a3 = 0;
  return r;
}

// RSYM (src/oprop.f90:2145-2200): folds the negative-wavenumber part of a
// grid of spacing dv starting at vft <= 0 onto the positive part, in place.
// R[i] is grid point i (its wavenumber vft + (i-1) dv); the loop reads R[0]
// and up to R[2 IP + 1] with IP <= 32, all inside the first panel's grids.
__device__ void rsym(double* R, double dv, double vft) {
  long ip = fint((-vft / dv) + 1. - .000001);
  ip = ip + 1;
  double P = (double(ip - 1) + vft / dv) * 2.;
  const double pst = P;
  if (P > 1.) P = P - 1.;
  const double wn1 = -P * (P - 1.) * (P - 2.) / 6.;
  const double w0 = (P * P - 1.) * (P - 2.) / 2.;
  const double w1 = -P * (P + 1.) * (P - 2.) / 2.;
  const double w2 = P * (P * P - 1.) / 6.;
  long k = ip;
  const long ipmax = ip + ip - 1;
  if (pst > 1.) {
    double b1 = R[ip - 2], b2 = R[ip - 1], c1 = R[k], c2;
    for (long i = ip; i <= ipmax; i++) {
      k = k - 1;
      c2 = c1;
      if (k < 1) return;
      c1 = R[k];
      R[k] = R[k] + wn1 * R[i + 1] + w0 * R[i] + w1 * b2 + w2 * b1;
      b1 = b2;
      b2 = R[i];
      if (k <= 2) continue;
      R[i] = R[i] + wn1 * c2 + w0 * c1 + w1 * R[k - 1] + w2 * R[k - 2];
    }
    return;
  }
  double c1 = R[ip], c2 = R[ip + 1], b2 = R[ip - 1], b1;
  for (long i = ip; i <= ipmax; i++) {
    k = k - 1;
    b1 = b2;
    b2 = R[i];
    if (k <= 1) return;
    R[i] = R[i] + wn1 * c2 + w0 * c1 + w1 * R[k] + w2 * R[k - 1];
    c2 = c1;
    c1 = R[k];
    R[k] = R[k] + wn1 * R[i + 2] + w0 * R[i + 1] + w1 * b2 + w2 * b1;
  }
}

// Candidate records of every panel: the layer's packed accepted lines whose
// centre lies within the layer's widest R3 half-window (+2 points) of the
// panel's R3 span; as ranks into the layer's packed list.
__global__ void k_panel_ranges(Work w, const int32_t* panel_layer, const int64_t* panel_base,
                               int64_t npanel_total, int64_t* rng) {
  const int64_t gp = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gp >= npanel_total) return;
  const int l = panel_layer[gp];
  const LayerDev& L = w.L[l];
  const PanelRange R = panel_range(L, (int32_t)(gp - panel_base[l]));
  const double reach = double(w.n_hw3[l] + 2) * L.dvr3;
  const double* v = w.n_rvnu + L.off_near;
  const int64_t n = w.n_cnt[l];
  rng[2 * gp] = lower_bound_d(v, 0, n, L.vft0 + double(R.a3 - 1) * L.dvr3 - reach);
  rng[2 * gp + 1] = lower_bound_d(v, 0, n, L.vft0 + double(R.b3 - 1) * L.dvr3 + reach);
}

// Warps of a 256-thread CTA whose threads own local points of [lo, hi]
// (clipped to [0, n)), thread t owning the points i with i mod 256 == t.
__device__ __forceinline__ uint32_t warps_of(int lo, int hi, int n) {
  lo = lo < 0 ? 0 : lo;
  hi = hi > n - 1 ? n - 1 : hi;
  if (hi < lo) return 0u;
  if (hi - lo >= 255) return 0xffu;
  const int a = (lo & 255) >> 5, b = (hi & 255) >> 5;
  const uint32_t up = 0xffu & ~((1u << a) - 1u), down = (2u << b) - 1u;
  return ((lo >> 8) == (hi >> 8)) ? (up & down) : ((up | down) & 0xffu);
}

constexpr int kPanelThreads = 256;
constexpr int kP1 = 10;           // R1 points per thread (2560 >= 2433)
constexpr int kP2 = 3;            // R2 points per thread (768 >= 611)
constexpr int kSegMax = kPanelSegMax;  // RADFNI segments kept per panel
constexpr int kSegCap = 64;       // segments a CTA builds at a time when a panel has more

// ---- bulk copies into shared memory, completed on an mbarrier -------------
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
// make the initialised barriers visible to the asynchronous proxy
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// order this thread's (and, after a CTA barrier, the CTA's) generic-proxy
// accesses of shared memory before later asynchronous-proxy writes
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// global -> shared bulk copy (no multicast); bytes a multiple of 16, both
// addresses 16-byte aligned
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for phase `parity` of a barrier, giving up after about a second.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
  for (int it = 0; it < (1 << 24); it++) {
    if (mbar_try_wait(bar, parity)) return true;
    if (it > 16) __nanosleep(64);
  }
  return false;
}

// Kahan-compensated FP32 accumulation of one grid point (sum, compensation).
__device__ __forceinline__ void kahan_add(float2& a, float v) {
  const float y = __fsub_rn(v, a.y);
  const float t = __fadd_rn(a.x, y);
  a.y = __fsub_rn(__fsub_rn(t, a.x), y);
  a.x = t;
}

// Line q's contribution at panel coordinate gi (= off + local point) of one
// grid, zc its centre on that grid: F1 + FG + VERFN terms on R1, F2 on R2,
// F3 on R3, with the line-coupling factor (:1322-1351).  T = double: FP64;
// T = float: the table index from the same FP64 position, the line shape in
// FP32.  The fused multiply-adds are written out, so that every panel
// variant rounds the shape alike wherever the compiler places this code.
template <typename T, int GRID>
__device__ __forceinline__ T near_val(const NearRec& q, const DevShapes& sh, int gi, double zc) {
  const double cf = GRID == 1 ? 4. / 2000. : (GRID == 2 ? 16. / 2000. : 64. / 2000.);
  const double zf = __dmul_rn(__dsub_rn(double(gi), zc), q.zslope);
  int iz = (int)(fabs(zf) + 1.5);
  iz = iz > kNfmx ? kNfmx : iz;
  if constexpr (sizeof(T) == 8) {
    double v;
    if (GRID == 1) {
      const double2 fab = *reinterpret_cast<const double2*>(sh.r1p + 4 * iz);
      v = fma(q.sx, sh.r1p[4 * iz + 2], fma(q.sg, fab.y, __dmul_rn(q.s0, fab.x)));
    } else {
      v = __dmul_rn(GRID == 2 ? q.s2 : q.s3, GRID == 2 ? sh.f2[iz] : sh.f3[iz]);
    }
    if (q.sppsp != 0.) v = fma(v, __dmul_rn(__dmul_rn(cf, q.sppsp), zf), v);
    return v;
  } else {
    float v;
    if (GRID == 1) {
      const float4 t = sh.r1p32[iz];
      v = fmaf((float)q.sx, t.z, fmaf((float)q.sg, t.y, __fmul_rn((float)q.s0, t.x)));
    } else {
      v = __fmul_rn((float)(GRID == 2 ? q.s2 : q.s3), GRID == 2 ? sh.f2_32[iz] : sh.f3_32[iz]);
    }
    const float cs = (float)__dmul_rn(cf, q.sppsp);
    if (cs != 0.f) v = fmaf(v, __fmul_rn(cs, (float)zf), v);
    return v;
  }
}

// Adds line q's contributions to the points this thread owns on one grid:
// local points [lo, hi] of the panel's span (thread tid owns tid + 256 k);
// `off` maps a local point to the line's panel coordinate.  T = double:
// FP64 sums; T = float: a Kahan-compensated FP32 sum.
template <typename T, int GRID>
__device__ __forceinline__ void near_add(const NearRec& q, const DevShapes& sh, int tid, int lo,
                                         int hi, int off, double zc, double* acc) {
  int i = tid + (lo > tid ? ((lo - tid + kPanelThreads - 1) / kPanelThreads) * kPanelThreads : 0);
  if constexpr (sizeof(T) == 8) {
#pragma unroll 2
    for (; i <= hi; i += kPanelThreads)
      acc[i] = __dadd_rn(acc[i], near_val<double, GRID>(q, sh, off + i, zc));
  } else {
    float2* a2 = reinterpret_cast<float2*>(acc);
#pragma unroll 2
    for (; i <= hi; i += kPanelThreads) kahan_add(a2[i], near_val<float, GRID>(q, sh, off + i, zc));
  }
}

// RADFNI segments of every panel (restarted each panel, src/oprop.f90:
// 2297-2475), one thread per panel: [start point, value, slope] each; a
// panel needing more than kSegMax keeps a count of -1 and builds its own.
__global__ void k_panel_segs(Work w, const int32_t* panel_layer, const int64_t* panel_base,
                             int64_t npanel_total, double* segs, int32_t* nseg) {
  const int64_t gp = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gp >= npanel_total) return;
  const int l = panel_layer[gp];
  const LayerDev& L = w.L[l];
  if (L.jrad != 0) return;
  const int64_t p = gp - panel_base[l];
  const long nhi = (p == L.npanel - 1) ? (long)(L.npts - 2400 * (L.npanel - 1) + 32) : 2432;
  const double DV = L.dv;
  const double vft = w.vft[L.off_panel + p];
  double vitst = vft + double(33 - 1) * DV - DV, rdlast = -1.;
  long n2 = 32;
  int ns = 0;
  double* out = segs + gp * (3 * kSegMax);
  do {
    const long n1 = n2 + 1;
    const double vi = vft + double(n1 - 1) * DV;
    double rdel;
    const double rv = radfni(vi, DV, L.xkt, vitst, rdel, rdlast);
    n2 = fint((vitst - vft) / DV + 0.001);
    if (n2 > nhi) n2 = nhi;
    if (ns == kSegMax) {
      ns = -1;
      break;
    }
    out[3 * ns] = double(n1);
    out[3 * ns + 1] = rv;
    out[3 * ns + 2] = rdel;
    ns++;
  } while (n2 < nhi);
  nseg[gp] = ns;
}

// PANEL (src/oprop.f90:1371-1561) fused with the near-wing sums, one CTA
// per panel: the panel's R1, R2 and R3 points are summed from its lines in
// file order (each thread owns fixed points, held in shared memory), R3
// gets the far wing and continuum by XINT (:515-519) and feeds R2 by
// 4-point interpolation, and the optical depth R1 + interpolated R2, times
// the radiation term, is written out.  The three grids never leave the SM.
//
// The panel's candidate lines (packed 96-byte records of the layer's
// accepted lines, in file order) arrive in batches of STAGE by bulk copies
// into a two-buffer ring: batch b+1 is in flight while the warps add batch
// b.  A warp visits only the records whose windows reach its points.
template <typename T, int STAGE, int MINB>
__global__ void __launch_bounds__(kPanelThreads, MINB)
    k_panel_od(Work w, DevShapes sh, const int32_t* panel_layer, const int64_t* panel_base,
               const int64_t* rng, const double* segs, const int32_t* nseg) {
  const int64_t gp = blockIdx.x;
  const int l = panel_layer[gp];
  const LayerDev& L = w.L[l];
  const int32_t p = (int32_t)(gp - panel_base[l]);
  const PanelRange R = panel_range(L, p);
  const int32_t n_r2 = (int32_t)L.n_r2;
  const int tid = threadIdx.x, warp = tid >> 5;
  __shared__ __align__(128) NearRec st[2][STAGE];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ __align__(16) double s1[kP1 * kPanelThreads];
  __shared__ __align__(16) double s2[kP2 * kPanelThreads];
  __shared__ __align__(16) double s3[kPanelThreads];
  __shared__ double seg[3 * kSegCap];  // [start, radvi, rdel] per segment
  __shared__ int s_nseg;
  __shared__ long s_n2;
  const int n1p = (int)(R.b1 - R.a1 + 1), n2p = (int)(R.b2 - R.a2 + 1),
            n3p = (int)(R.b3 - R.a3 + 1);
  const int lane = tid & 31;
  const int64_t clo = rng[2 * gp], chi = rng[2 * gp + 1];
  const NearRec* src = w.n_rec + L.off_near;
  const int nbatch = (int)((chi - clo + STAGE - 1) / STAGE);
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
  }
  __syncthreads();
  auto issue = [&](int b) {  // thread 0: batch b into buffer b & 1
    const int64_t c0 = clo + (int64_t)b * STAGE;
    const int n = (int)((chi - c0) < STAGE ? (chi - c0) : STAGE);
    const unsigned bytes = (unsigned)n * (unsigned)sizeof(NearRec);
    mbar_expect_tx(&bar[b & 1], bytes);
    bulk_g2s(st[b & 1], src + c0, bytes, &bar[b & 1]);
  };
  if (tid == 0 && nbatch > 0) issue(0);
  // the grids start at zero (FP32: sum and compensation pairs)
  {
    double2* z1 = reinterpret_cast<double2*>(s1);
    double2* z2 = reinterpret_cast<double2*>(s2);
    for (int i = tid; i < kP1 * kPanelThreads / 2; i += kPanelThreads) z1[i] = make_double2(0., 0.);
    for (int i = tid; i < kP2 * kPanelThreads / 2; i += kPanelThreads) z2[i] = make_double2(0., 0.);
    s3[tid] = 0.;
  }
  int lost = -1;  // batch whose copy did not complete
  for (int b = 0; b < nbatch; b++) {
    // buffer (b+1)&1 was last read in batch b-1, which every thread has
    // finished (barrier at the end of that batch)
    if (tid == 0 && b + 1 < nbatch) {
      fence_proxy_async_smem();
      issue(b + 1);
    }
    if (!mbar_wait_bounded(&bar[b & 1], (unsigned)((b >> 1) & 1))) {
      lost = b;
      break;
    }
    const int64_t c0 = clo + (int64_t)b * STAGE;
    const int n = (int)((chi - c0) < STAGE ? (chi - c0) : STAGE);
    const NearRec* batch = st[b & 1];
    // Thread t owns local points t + 256 j of each grid.  Lane k of every
    // warp tests record k0+k, one ballot per grid gives the records whose
    // clipped window reaches the warp's points, and the warp adds those in
    // file order.
    for (int k0 = 0; k0 < n; k0 += 32) {
      const int k = k0 + lane;
      const NearRec& qk = batch[k < n ? k : 0];
      // R1 (DV grid): F1 + FG + VERFN terms
      unsigned m = __ballot_sync(
          0xffffffffu, k < n && ((warps_of(qk.lo1 - R.a1, qk.hi1 - R.a1, n1p) >> warp) & 1u));
      while (m) {
        const NearRec& q = batch[k0 + __ffs(m) - 1];
        m &= m - 1;
        near_add<T, 1>(q, sh, tid, max(q.lo1, R.a1) - R.a1, min(q.hi1, R.b1) - R.a1,
                       R.a1 - 2400 * q.pc - 1, q.zint, s1);
      }
      // R2 (4 DV): F2
      m = __ballot_sync(
          0xffffffffu, k < n && ((warps_of(qk.lo2 - R.a2, qk.hi2 - R.a2, n2p) >> warp) & 1u));
      while (m) {
        const NearRec& q = batch[k0 + __ffs(m) - 1];
        m &= m - 1;
        near_add<T, 2>(q, sh, tid, max(q.lo2, R.a2) - R.a2, min(q.hi2, R.b2) - R.a2,
                       R.a2 - 600 * q.pc - 1, q.zint * L.conf2, s2);
      }
      // R3 (16 DV): F3
      m = __ballot_sync(
          0xffffffffu, k < n && ((warps_of(qk.lo3 - R.a3, qk.hi3 - R.a3, n3p) >> warp) & 1u));
      while (m) {
        const NearRec& q = batch[k0 + __ffs(m) - 1];
        m &= m - 1;
        near_add<T, 3>(q, sh, tid, max(q.lo3, R.a3) - R.a3, min(q.hi3, R.b3) - R.a3,
                       R.a3 - 150 * q.pc - 1, q.zint * L.conf3, s3);
      }
    }
    __syncthreads();
  }
  if (lost >= 0) {
    // a bulk copy did not complete: flag it, give the copies in flight
    // (that batch and the next) another bounded wait, and leave the panel
    // unwritten
    if (tid == 0) atomicExch(&w.status[0], 4);
    mbar_wait_bounded(&bar[lost & 1], (unsigned)((lost >> 1) & 1));
    if (lost + 1 < nbatch) mbar_wait_bounded(&bar[(lost + 1) & 1], (unsigned)(((lost + 1) >> 1) & 1));
    return;
  }
  if constexpr (sizeof(T) == 4) {
    // compensated FP32 sums to FP64, each thread its own points in place
    for (int i = tid; i < kP1 * kPanelThreads; i += kPanelThreads) {
      const float2 a = reinterpret_cast<const float2*>(s1)[i];
      s1[i] = (double)a.x - (double)a.y;
    }
    for (int i = tid; i < kP2 * kPanelThreads; i += kPanelThreads) {
      const float2 a = reinterpret_cast<const float2*>(s2)[i];
      s2[i] = (double)a.x - (double)a.y;
    }
    {
      const float2 a = reinterpret_cast<const float2*>(s3)[tid];
      s3[tid] = (double)a.x - (double)a.y;
    }
    __syncthreads();
  }
  // RSYM on the three grids of a first panel starting at or below zero
  // (HIRAC1 :501-505), before the far wing and continuum are added
  if (R.a1 == 0) {
    __syncthreads();  // the grids are complete (also when no line reached the panel)
    if (tid == 0) {
      const double vft = w.vft[L.off_panel];
      rsym(s1, L.dv, vft);
      rsym(s2, L.dvr2, vft);
      rsym(s3, L.dvr3, vft);
    }
    __syncthreads();
  }
  // R3 += XINT(R4 of the owning panel's window) + XINT(ABSRB): R3 point g
  // belongs to panel 0 for g <= 155, else to panel (g-6)/150 (N1R3/N2R3,
  // src/oprop.f90:474-486)
  if (tid < n3p) {
    const int32_t g = R.a3 + tid;
    const int32_t po = (g <= 155) ? 0 : (g - 6) / 150;
    if (po < L.npanel) {
      const long I = (long)(g - 150 * po);
      const long n1 = (po == 0) ? 1 : 6;
      const double vft = w.vft[L.off_panel + po];
      double add = 0.;
      if (L.ilblf4 >= 1 && L.nwin > 0) {
        const int wi = w.win_of[L.off_panel + po];
        const WinDev& W = w.win[L.off_win + wi];
        add += xint_at(W.v1r4, W.v2r4, L.dvr4, w.r4 + (L.off_win + wi) * kR4Stride, vft, L.dvr3,
                       I, n1, 155);
      }
      if (L.icntnm >= 1)
        add += xint_at(L.v1abs, L.v2abs, L.dvabs, w.absrb + L.off_abs, vft, L.dvr3, I, n1, 155);
      s3[tid] += add;
    }
  }
  __syncthreads();
  // R2 += 4-point interpolation of R3 (PANEL :1459-1480)
  for (int i = tid; i < n2p; i += kPanelThreads) {
    const int32_t g = R.a2 + i;
    if (g >= 5 && g <= n_r2 - 3) s2[i] += interp4(s3 - R.a3, (g - 1) / 4 + 1, (g - 1) % 4);
  }
  __syncthreads();
  // OD = R1 + 4-point interpolation of R2 (PANEL :1482-1519), times the
  // radiation term, piecewise linear over the panel's RADFNI segments
  double* od_out = w.od + L.off_od;
  const double* r2 = s2 - R.a2;
  if (L.jrad != 0) {
    for (int i = tid; i < n1p; i += kPanelThreads) {
      const int32_t g = R.a1 + i;
      if (g < 33) continue;  // below V1: a folded first panel's lower points
      od_out[g - 33] = s1[i] + interp4(r2, (g - 1) / 4 + 1, (g - 1) % 4);
    }
    return;
  }
  const int nsg = nseg[gp];
  const double* sgp = segs + gp * (3 * kSegMax);
  // thread 0's RADFNI state when the panel builds its own segments
  double vitst = 0., rdlast = -1.;
  long n2 = 32;
  const double DV = L.dv;
  const double vft = w.vft[L.off_panel + p];
  if (tid == 0) vitst = vft + double(33 - 1) * DV - DV;
  for (;;) {
    if (nsg >= 0) {
      for (int k = tid; k < 3 * nsg; k += kPanelThreads) seg[k] = sgp[k];
      if (tid == 0) {
        s_nseg = nsg;
        s_n2 = R.nhi;
      }
    } else if (tid == 0) {
      int ns = 0;
      do {
        const long n1 = n2 + 1;
        const double vi = vft + double(n1 - 1) * DV;
        double rdel;
        const double rv = radfni(vi, DV, L.xkt, vitst, rdel, rdlast);
        n2 = fint((vitst - vft) / DV + 0.001);
        if (n2 > R.nhi) n2 = R.nhi;
        seg[3 * ns] = double(n1);
        seg[3 * ns + 1] = rv;
        seg[3 * ns + 2] = rdel;
        ns++;
      } while (n2 < R.nhi && ns < kSegCap);
      s_nseg = ns;
      s_n2 = n2;
    }
    __syncthreads();
    const int ns = s_nseg;
    const int32_t ilo = (int32_t)seg[0], ihi = (int32_t)s_n2;
    int lo = 0;  // this thread's segment: its points only increase
    for (int i = tid; i < n1p; i += kPanelThreads) {
      const int32_t g = R.a1 + i;
      const int32_t I = g - 2400 * p;
      if (I < ilo || I > ihi || g < 33) continue;
      double od = s1[i] + interp4(r2, (g - 1) / 4 + 1, (g - 1) % 4);
      while (lo + 1 < ns && seg[3 * (lo + 1)] <= double(I)) lo++;
      od = od * (seg[3 * lo + 1] + double(I - (int32_t)seg[3 * lo]) * seg[3 * lo + 2]);
      od_out[g - 33] = od;
    }
    if (ihi >= R.nhi) break;
    __syncthreads();  // the next batch overwrites the segments
  }
}

// =========================================================================
// XMERGE for one layer: EMIN (src/xmerge.f90:1795-1855) then EMINIT
// (:2436-2484) for the first layer or RADNN IPATH=1 (:2985-3130) after.
// =========================================================================
// Planck function in the arithmetic T, from an FP64 wavenumber.
template <typename T>
__device__ __forceinline__ T planck_t(double vi, double xkt, double rk) {
  if constexpr (sizeof(T) == 8) {
    return planck(vi, xkt, rk);
  } else {
    if (!(xkt > 0.0)) return 0.f;
    const float x = (float)(vi * rk);
    const float v = (float)vi;
    float b = 0.f;
    if (x < 1e-2f) b = (v * v) * (float)xkt / (1.f + 0.5f * x);
    else if (x <= 80.f) b = (v * v * v) / expm1f(x);
    return b * (float)kRADCN1;
  }
}

// EMIN at one point (src/xmerge.f90:1795-1855): the layer's transmittance
// and linear-in-tau emission.  The source function's weight
// F = 1 - 2 (T/(T-1) + 1/tau) is taken over one common denominator.
template <typename T>
__device__ __forceinline__ void emin_point(double odv, double vi, const EminT& t, T& tr, T& em) {
  T o = (T)odv;
  if (o < (T)-kODLO) o = (T)-kODLO;
  tr = exp(-o);
  const T d = tr - (T)1.;
  const T fi = (o <= (T)kODLO) ? o * (T)(1. / 6.) : (T)1. - (T)2. * ((tr * o + d) / (d * o));
  const T bb = planck_t<T>(vi, t.xkt, t.rk);
  const T bbd = (t.xkta > 0.) ? planck_t<T>(vi, t.xkta, t.rka) - bb : (T)0.;
  em = ((T)1. - tr) * (bb + bbd * fi);
}

// EMIN at one point for the symmetric tangent path (XKTB > 0, specular,
// src/xmerge.f90:1984-2019): the emission of the layer's near crossing (the
// level term at XKTA) and of its far crossing (the level term at XKTB).
template <typename T>
__device__ __forceinline__ void emin_point_b(double odv, double vi, const EminT& t, double xktb,
                                             double rkb, T& tr, T& em, T& emb) {
  T o = (T)odv;
  if (o < (T)-kODLO) o = (T)-kODLO;
  tr = exp(-o);
  const T d = tr - (T)1.;
  const T fi = (o <= (T)kODLO) ? o * (T)(1. / 6.) : (T)1. - (T)2. * ((tr * o + d) / (d * o));
  const T bb = planck_t<T>(vi, t.xkt, t.rk);
  const T bba = (t.xkta > 0.) ? planck_t<T>(vi, t.xkta, t.rka) - bb : (T)0.;
  const T bbb = (xktb > 0.) ? planck_t<T>(vi, xktb, rkb) - bb : (T)0.;
  const T ab = (T)1. - tr;
  em = ab * (bb + bba * fi);
  emb = ab * (bb + bbb * fi);
}

// emin_point in FP64 with the three divisions (two Planck quotients
// e/(1-e) and the source weight's common denominator) taken from one
// reciprocal of their product; differs from emin_point by a few units in
// the last place.
__device__ __forceinline__ void emin_point_1div(double odv, double vi, const EminT& t, double& tr,
                                                double& em) {
  double o = odv;
  if (o < -kODLO) o = -kODLO;
  tr = exp(-o);
  const double d = tr - 1.;
  const bool lin = o <= kODLO;
  // Planck: the main branch needs e/(1-e) with e = exp(-x)
  auto pre = [&](double xkt, double rk, double& e, double& small, int& br) {
    br = 0;  // 0: zero, 1: small-x form, 2: main
    e = 0.;
    small = 0.;
    if (xkt > 0.0) {
      const double x = vi * rk;
      if (x < 1e-2) {
        br = 1;
        small = (vi * vi) * xkt / (1. + 0.5 * x);
      } else if (x <= 80.) {
        br = 2;
        e = exp(-x);
      }
    }
  };
  double e1, s1, e2, s2;
  int b1, b2;
  pre(t.xkt, t.rk, e1, s1, b1);
  const bool bnd = t.xkta > 0.;
  if (bnd) pre(t.xkta, t.rka, e2, s2, b2);
  else b2 = 0, e2 = 0., s2 = 0.;
  const double D1 = b1 == 2 ? 1. - e1 : 1.;
  const double D2 = b2 == 2 ? 1. - e2 : 1.;
  const double D3 = lin ? 1. : d * o;
  const double r = 1. / ((D1 * D2) * D3);
  const double v3 = (vi * vi) * vi;
  const double bb = kRADCN1 * (b1 == 2 ? v3 * e1 * ((D2 * D3) * r) : s1);
  const double bt = kRADCN1 * (b2 == 2 ? v3 * e2 * ((D1 * D3) * r) : s2);
  const double bbd = bnd ? bt - bb : 0.;
  const double fi = lin ? o * (1. / 6.) : 1. - 2. * ((tr * o + d) * ((D1 * D2) * r));
  em = (1. - tr) * (bb + bbd * fi);
}

// emin_point_1div with the two Planck exponentials e1 = exp(-vi*rk) and
// e2 = exp(-vi*rka) supplied by the caller (used only where the main
// Planck branch applies).
__device__ __forceinline__ void emin_point_e(double odv, double vi, const EminT& t, double e1,
                                             double e2, double& tr, double& em) {
  double o = odv;
  if (o < -kODLO) o = -kODLO;
  tr = exp(-o);
  const double d = tr - 1.;
  const bool lin = o <= kODLO;
  auto branch = [&](double xkt, double rk, double& small) {
    small = 0.;
    if (!(xkt > 0.0)) return 0;
    const double x = vi * rk;
    if (x < 1e-2) {
      small = (vi * vi) * xkt / (1. + 0.5 * x);
      return 1;
    }
    return x <= 80. ? 2 : 0;
  };
  double s1, s2 = 0.;
  const int b1 = branch(t.xkt, t.rk, s1);
  const bool bnd = t.xkta > 0.;
  const int b2 = bnd ? branch(t.xkta, t.rka, s2) : 0;
  const double D1 = b1 == 2 ? 1. - e1 : 1.;
  const double D2 = b2 == 2 ? 1. - e2 : 1.;
  const double D3 = lin ? 1. : d * o;
  const double r = 1. / ((D1 * D2) * D3);
  const double v3 = (vi * vi) * vi;
  const double bb = kRADCN1 * (b1 == 2 ? v3 * e1 * ((D2 * D3) * r) : s1);
  const double bt = kRADCN1 * (b2 == 2 ? v3 * e2 * ((D1 * D3) * r) : s2);
  const double bbd = bnd ? bt - bb : 0.;
  const double fi = lin ? o * (1. / 6.) : 1. - 2. * ((tr * o + d) * ((D1 * D2) * r));
  em = (1. - tr) * (bb + bbd * fi);
}

// Point f of the finer grid from the previous layer's field x (n_old
// points): a copy where the grids agree, else RADNN's 4-point Lagrange
// interpolation at P = 1 - r/(ITYPE+1) (ITYPE = DV/(DV_old-DV) rounded).
// 32-bit indices: layers hold fewer than 2^31 points.
__device__ __forceinline__ void merge_regrid(const double* x, const double* y, int32_t n_old,
                                             int32_t f, int32_t itype, double& xo, double& yo) {
  auto cl = [&](int32_t c) { return c < 0 ? 0 : (c >= n_old ? n_old - 1 : c); };
  if (itype == 0) {
    xo = x[cl(f)];
    if (y) yo = y[cl(f)];
    return;
  }
  const int32_t LL = itype + 1;
  const int32_t q = f / LL, r = f - q * LL;
  if (r == 0) {
    xo = x[cl(q * itype)];
    if (y) yo = y[cl(q * itype)];
    return;
  }
  const int32_t ipl = q * itype + r - 1;
  const double P = 1.0 - double(r) / double(LL);
  const double a1 = -P * (P - 1.0) * (P - 2.0) / 6.0, a2 = (P * P - 1.0) * (P - 2.0) * 0.5;
  const double a3 = -P * (P + 1.0) * (P - 2.0) * 0.5, a4 = P * (P * P - 1.0) / 6.0;
  const int32_t c0 = cl(ipl - 1), c1 = cl(ipl), c2 = cl(ipl + 1), c3 = cl(ipl + 2);
  xo = a1 * x[c0] + a2 * x[c1] + a3 * x[c2] + a4 * x[c3];
  if (y) yo = a1 * y[c0] + a2 * y[c1] + a3 * y[c2] + a4 * y[c3];
}

// ABSMRG's regrid of the accumulated optical depth (src/xmerge.f90:437-682):
// the interpolation of merge_regrid, except at the end of the old field.
// ABSMRG advances its old-point counter NVS with every new point (label
// 190); once NVS passes the old field's last point but two and no old data
// is left, every later point takes the mean of the last two old points
// (label 210).  Point f-1 used NVS = q*ITYPE + max(r, 1) (q, r = (f-1) divided
// by ITYPE+1), and NVS never decreases, so point f lies in that tail when
// NVS of point f-1 has reached n_old-2.
__device__ __forceinline__ double absmrg_regrid(const double* x, int32_t n_old, int32_t f,
                                                int32_t itype) {
  if (itype > 0 && f >= 2 && n_old >= 2) {
    const int32_t g = f - 1, LL = itype + 1;
    const int32_t q = g / LL, r = g - q * LL;
    const int32_t nvs = q * itype + (r > 1 ? r : 1);
    if (nvs >= n_old - 2) return (x[n_old - 1] + x[n_old - 2]) * 0.5;
  }
  double xo = 0., unused = 0.;
  merge_regrid(x, nullptr, n_old, f, itype, xo, unused);
  return xo;
}

template <typename T>
__global__ void k_merge(const LayerDev* Lp, const double* vft_panel, const double* od,
                        int first, double dv_old, int64_t n_old64, const double* rad_in,
                        const double* tr_in, double* rad_out, double* tr_out, double tbnd,
                        double emis, int iemit, double tzu, int down, double tbnd_last,
                        double tzl_b, double refl) {
  const LayerDev& L = *Lp;
  const int32_t f = (int32_t)(blockIdx.x * blockDim.x + threadIdx.x);
  if (f >= (int32_t)L.npts) return;
  const int32_t n_old = (int32_t)n_old64;
  const double DV = L.dv;
  const int32_t p = f / 2400;
  const double vi = (vft_panel[p] + double(33 - 1) * DV) + double(f - 2400 * p) * DV;
  const double odv = od[f];
  const int32_t itype = (first || dv_old == DV) ? 0 : (int32_t)fint(DV / (dv_old - DV) + 0.5);
  if (iemit == 0) {
    // ABINIT / ABSMRG: optical depths add
    const double old = first ? 0. : absmrg_regrid(rad_in, n_old, f, itype);
    rad_out[f] = odv + old;
    if (tr_out) tr_out[f] = 0.;
    return;
  }
  T tr, em;
  if (tzl_b > 0.) {
    // the symmetric tangent path (IPATHL=2, IANT=0: EMINIT :2442-2447,
    // RADNN IPATH=2 :2997-3005, 3132-3148) or, with refl > 0, the reflected
    // atmosphere (IPATHL=-1, specular: EMINIT :2486-2540, RADNN IPATH=-10
    // :3051-3066, 3197-3215); EMB is the emission at the lower level's
    // temperature
    T emb;
    emin_point_b<T>(odv, vi, emin_temps(L.tave, tzu), tzl_b / kRADCN2, kRADCN2 / tzl_b, tr, em,
                    emb);
    const double trd = (double)tr, emd = (double)em, embd = (double)emb;
    if (first) {
      if (refl > 0.) {
        const double bb = tbnd > 0. ? planck(vi, tbnd / kRADCN2, kRADCN2 / tbnd) : 0.;
        rad_out[f] = emd + embd * refl * trd + trd * bb * emis;
        tr_out[f] = trd;
      } else {
        rad_out[f] = emd + embd * trd;
        tr_out[f] = trd * trd;
      }
      return;
    }
    double ro, to;
    merge_regrid(rad_in, tr_in, n_old, f, itype, ro, to);
    const double tt = trd * to;
    if (refl > 0.) {
      rad_out[f] = trd * ro + emd + embd * to * tt * refl;
      tr_out[f] = tt;
    } else {
      rad_out[f] = trd * ro + emd + embd * tt;
      tr_out[f] = trd * tt;
    }
    return;
  }
  emin_point<T>(odv, vi, emin_temps(L.tave, tzu), tr, em);
  if (first) {
    // EMINIT: boundary emission (:2436-2484)
    if (tbnd > 0.) em = em + tr * planck_t<T>(vi, tbnd / kRADCN2, kRADCN2 / tbnd) * (T)emis;
    rad_out[f] = (double)em;
    tr_out[f] = (double)tr;
    return;
  }
  // RADNN: IPATH=1, R = T_layer R_old + E; IPATH=3 (looking up), R = R_old +
  // E T_old; T = T_layer T_old
  double ro, to;
  merge_regrid(rad_in, tr_in, n_old, f, itype, ro, to);
  double rn = down ? ro + (double)em * to : (double)tr * ro + (double)em;
  const double tn = (double)tr * to;
  // EMBND (:3652-3733) beyond the last layer looking up
  if (tbnd_last > 0.)
    rn = rn + tn * emis * (double)planck_t<T>(vi, tbnd_last / kRADCN2, kRADCN2 / tbnd_last);
  rad_out[f] = rn;
  tr_out[f] = tn;
}

// k_merge over m.nl consecutive layers on one grid (in FP64 with EMIN's
// quotients from one reciprocal, emin_point_1div); the next layer's optical
// depth is fetched while this one merges.  DOWN: looking up (m.down).
template <typename T, bool DOWN>
__global__ void __launch_bounds__(256) k_merge_run(const MergeRun m, const double* vft_panel,
                                                   const double* od, int32_t f_lo, int32_t f_hi,
                                                   double DV, const double* rad_in,
                                                   const double* tr_in, double* rad_out,
                                                   double* tr_out, double tbnd, double emis,
                                                   int iemit) {
  const int32_t f = f_lo + (int32_t)(blockIdx.x * blockDim.x + threadIdx.x);
  if (f >= f_hi) return;
  const int32_t p = f / 2400;
  const double vi = (vft_panel[p] + double(33 - 1) * DV) + double(f - 2400 * p) * DV;
  double ro = 0., to = 1.;
  if (!m.first) {
    if (iemit) merge_regrid(rad_in, tr_in, m.n_old, f, m.itype, ro, to);
    else ro = absmrg_regrid(rad_in, m.n_old, f, m.itype);
  }
  double odn = od[m.od_off[0] + f];
  for (int l = 0; l < m.nl; l++) {
    const double odv = odn;
    if (l + 1 < m.nl) odn = od[m.od_off[l + 1] + f];
    if (iemit == 0) {
      ro = (m.first && l == 0) ? odv : odv + ro;
      continue;
    }
    T tr, em;
    if (!DOWN && (m.tangent || m.refl > 0.)) {
      // the symmetric tangent path (EMINIT :2442-2447, RADNN IPATH=2
      // :2997-3005, 3132-3148) and the reflected atmosphere (EMINIT
      // :2486-2540, RADNN IPATH=-10 :3051-3066, 3197-3215)
      T emb;
      emin_point_b<T>(odv, vi, m.t[l], m.tb_xkt[l], m.tb_rk[l], tr, em, emb);
      const double trd = (double)tr, emd = (double)em, embd = (double)emb;
      if (m.first && l == 0) {
        if (m.refl > 0.) {
          const double bb = tbnd > 0. ? planck(vi, tbnd / kRADCN2, kRADCN2 / tbnd) : 0.;
          ro = emd + embd * m.refl * trd + trd * bb * emis;
          to = trd;
        } else {
          ro = emd + embd * trd;
          to = trd * trd;
        }
      } else {
        const double tt = trd * to;
        if (m.refl > 0.) {
          ro = trd * ro + emd + embd * to * tt * m.refl;
          to = tt;
        } else {
          ro = trd * ro + emd + embd * tt;
          to = trd * tt;
        }
      }
      continue;
    }
    if constexpr (sizeof(T) == 8) emin_point_1div(odv, vi, m.t[l], tr, em);
    else emin_point<T>(odv, vi, m.t[l], tr, em);
    if (m.first && l == 0) {
      if (tbnd > 0.) em = em + tr * planck_t<T>(vi, tbnd / kRADCN2, kRADCN2 / tbnd) * (T)emis;
      ro = (double)em;
      to = (double)tr;
    } else if (DOWN) {
      // RADNN IPATH=3 (:3007-3013, 3150-3166): the farther layer's emission
      // seen through the nearer layers
      ro = ro + (double)em * to;
      to = (double)tr * to;
    } else {
      ro = (double)tr * ro + (double)em;
      to = (double)tr * to;
    }
  }
  // EMBND (:3652-3733) beyond the last layer looking up (XMERGE :140, 157)
  if (DOWN && iemit && m.tbnd_last > 0.)
    ro = ro + to * emis * (double)planck_t<T>(vi, m.tbnd_last / kRADCN2, kRADCN2 / m.tbnd_last);
  rad_out[f] = ro;
  if (tr_out) tr_out[f] = iemit ? to : 0.;
}

// k_merge_run in FP64 with MK points per thread, 256 apart (coalesced).
// The Planck exponentials of a layer follow the points as a geometric
// sequence: exp(-vi*rk) at the thread's first point, then one product by
// exp(-256*DV*rk) per point (s_st1/s_st2, one per layer); the points'
// wavenumbers differ from v + 256*j*DV only by the rounding of the panel
// origins, a relative change of the exponential far below 1e-13.  Per point
// and layer this leaves one exponential (the transmittance) and one
// reciprocal.
constexpr int kMergeThreads = 256;
constexpr int kMergePointsPerThread = 2;
template <bool DOWN, int MK>
__global__ void __launch_bounds__(kMergeThreads, 3) k_merge_run_f64(
    const MergeRun m, const double* vft_panel, const double* od, int32_t f_lo, int32_t f_hi,
    double DV, const double* rad_in, const double* tr_in, double* rad_out, double* tr_out,
    double tbnd, double emis, int iemit) {
  __shared__ double s_st1[kMergeRunMax], s_st2[kMergeRunMax];
  const int tid = threadIdx.x;
  if (tid < m.nl) {
    const EminT& t = m.t[tid];
    const double span = double(kMergeThreads) * DV;
    s_st1[tid] = t.xkt > 0. ? exp(-span * t.rk) : 0.;
    s_st2[tid] = t.xkta > 0. ? exp(-span * t.rka) : 0.;
  }
  __syncthreads();
  // groups of MK*256 points at absolute positions (a multiple of MK*256),
  // so that a point's arithmetic does not depend on the launch's range
  const int32_t g0 = (f_lo / (kMergeThreads * MK)) * (kMergeThreads * MK);
  const int32_t f0 = g0 + (int32_t)blockIdx.x * (kMergeThreads * MK) + tid;
  if (f0 >= f_hi) return;
  double vi[MK], ro[MK], to[MK], odn[MK];
#pragma unroll
  for (int j = 0; j < MK; j++) {
    const int32_t f = f0 + j * kMergeThreads;
    // clamped into the range: loads stay in range (the group's first point
    // is always a valid grid point, for its wavenumber)
    const int32_t fc = f < f_lo ? f_lo : (f < f_hi ? f : f_hi - 1);
    const int32_t fv = j == 0 ? f : fc;
    const int32_t p = fv / 2400;
    vi[j] = (vft_panel[p] + double(33 - 1) * DV) + double(fv - 2400 * p) * DV;
    ro[j] = 0.;
    to[j] = 1.;
    if (!m.first) {
      if (iemit) merge_regrid(rad_in, tr_in, m.n_old, fc, m.itype, ro[j], to[j]);
      else ro[j] = absmrg_regrid(rad_in, m.n_old, fc, m.itype);
    }
    odn[j] = od[m.od_off[0] + fc];
  }
  for (int l = 0; l < m.nl; l++) {
    double odv[MK];
#pragma unroll
    for (int j = 0; j < MK; j++) {
      odv[j] = odn[j];
      if (l + 1 < m.nl) {
        const int32_t f = f0 + j * kMergeThreads;
        odn[j] = od[m.od_off[l + 1] + (f < f_lo ? f_lo : (f < f_hi ? f : f_hi - 1))];
      }
    }
    if (iemit == 0) {
#pragma unroll
      for (int j = 0; j < MK; j++) ro[j] = (m.first && l == 0) ? odv[j] : odv[j] + ro[j];
      continue;
    }
    const EminT t = m.t[l];
    double e1 = t.xkt > 0. ? exp(-(vi[0] * t.rk)) : 0.;
    double e2 = t.xkta > 0. ? exp(-(vi[0] * t.rka)) : 0.;
    const double st1 = s_st1[l], st2 = s_st2[l];
#pragma unroll
    for (int j = 0; j < MK; j++) {
      if (j > 0) {
        e1 *= st1;
        e2 *= st2;
      }
      double tr, em;
      emin_point_e(odv[j], vi[j], t, e1, e2, tr, em);
      if (m.first && l == 0) {
        if (tbnd > 0.) em = em + tr * planck(vi[j], tbnd / kRADCN2, kRADCN2 / tbnd) * emis;
        ro[j] = em;
        to[j] = tr;
      } else if (DOWN) {
        ro[j] = ro[j] + em * to[j];
        to[j] = tr * to[j];
      } else {
        ro[j] = tr * ro[j] + em;
        to[j] = tr * to[j];
      }
    }
  }
#pragma unroll
  for (int j = 0; j < MK; j++) {
    const int32_t f = f0 + j * kMergeThreads;
    if (f >= f_hi) break;
    if (f < f_lo) continue;
    double r = ro[j];
    if (DOWN && iemit && m.tbnd_last > 0.)
      r = r + to[j] * emis * planck(vi[j], m.tbnd_last / kRADCN2, kRADCN2 / m.tbnd_last);
    rad_out[f] = r;
    if (tr_out) tr_out[f] = iemit ? to[j] : 0.;
  }
}

// =========================================================================
// Radiance Jacobians (the reference's analytic-Jacobian path, EMDT/EMADMG
// src/xmerge.f90:4406-5782 with TDERIVup/QDERIVup :5786-6144): the forward
// merge of one layer together with the derivative of that layer's merged
// radiance with respect to each parameter p,
//   d_p = dR/dtau * dtau/dp  +  [p = T] dE/dB * dB/dT
// where dtau/dp comes from optical depths at perturbed parameters (the
// reference's own layer-derivative route) and the rest is differentiated
// by hand.  All FP64.
// =========================================================================
constexpr int kJacMaxPar = 8;

// dB/dT of PLANCK (src/xmerge.f90:968-1017) at temperature t, both branches
__device__ __forceinline__ double planck_dt(double vi, double t) {
  if (!(t > 0.)) return 0.;
  const double xkt = t / kRADCN2;
  const double x = vi / xkt;
  if (x < 1e-2) return kRADCN1 * (vi * vi) / kRADCN2 * (1. + x) / ((1. + 0.5 * x) * (1. + 0.5 * x));
  if (x > 80.) return 0.;
  const double e = exp(-x);
  return kRADCN1 * (vi * vi * vi) * e / (1. - e) * (x / t) / (1. - e);
}

// PLANCK_DT (src/xmerge.f90:1019-1080): the factor of the Planck function's
// temperature derivative at XKT, times BBVAL (EMDT passes the layer's Planck
// value for both the layer and the upper level).
__device__ __forceinline__ double planck_dt_ref(double vi, double xkt, double bbval) {
  double v = 0.;
  if (xkt > 0.0) {
    const double viokt = vi / xkt, vtkelv = xkt * kRADCN2;
    if (viokt <= 1e-2) v = 1. / (-vtkelv * (1. + 5e-1 * viokt));
    else if (viokt <= 80.0) v = viokt / (vtkelv * (1. - exp(-viokt)));
  }
  return v * bbval;
}

struct JacRows {
  double* d[kJacMaxPar];        // per parameter: this layer's row
  const double* dtau[kJacMaxPar];  // per parameter: dtau/dp of this layer (mode 0) or
                                   // the perturbed run's optical depth (mode 1)
  int np;
  int mode;                     // 0: exact merge derivative; 1: TDERIVup/QDERIVup
  int k0;                       // parameter of row 0 (0: temperature)
};

__global__ void k_jac_layer(const LayerDev* Lp, const double* vft_panel, const double* od,
                            int first, double dv_old, int64_t n_old, const double* rad_in,
                            const double* tr_in, double* rad_out, double* tr_out, double tbnd,
                            double emis, double tzu, JacRows rows) {
  const LayerDev& L = *Lp;
  const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= L.npts) return;
  const double DV = L.dv;
  const int64_t p = f / 2400;
  const double vi = (vft_panel[p] + double(33 - 1) * DV) + double(f - 2400 * p) * DV;
  const EminT t = emin_temps(L.tave, tzu);
  const double xkta = t.xkta;
  const double tau = od[f];
  const bool clamped = tau < -kODLO;
  const double o = clamped ? -kODLO : tau;
  const double tr = exp(-o);
  double fi, dfi;
  if (o <= kODLO) {
    fi = o / 6.;
    dfi = 1. / 6.;
  } else {
    const double d = tr - 1.;
    fi = 1. - 2. * ((tr * o + d) / (d * o));
    dfi = -2. * (tr / (d * d) - 1. / (o * o));
  }
  const double bb = planck(vi, t.xkt, t.rk);
  const double bbd = (xkta > 0.) ? planck(vi, xkta, t.rka) - bb : 0.;
  const double em = (1. - tr) * (bb + bbd * fi);
  const double dem_do = tr * (bb + bbd * fi) + (1. - tr) * bbd * dfi;
  const double dem_db = (1. - tr) * (xkta > 0. ? 1. - fi : 1.);
  double rad, trn, dr_do, rado;
  if (first) {
    const double bs = tbnd > 0. ? planck(vi, tbnd / kRADCN2, kRADCN2 / tbnd) * emis : 0.;
    rad = em + tr * bs;
    trn = tr;
    dr_do = dem_do - tr * bs;
    rado = bs;
  } else {
    const long itype = (dv_old == DV) ? 0 : fint(DV / (dv_old - DV) + 0.5);
    double ro, to;
    auto R = [&](int64_t c) { return rad_in[c < 0 ? 0 : (c >= n_old ? n_old - 1 : c)]; };
    auto TR = [&](int64_t c) { return tr_in[c < 0 ? 0 : (c >= n_old ? n_old - 1 : c)]; };
    const int64_t LL = itype + 1;
    const int64_t q = f / LL, r = f % LL;
    if (itype == 0) {
      ro = R(f);
      to = TR(f);
    } else if (r == 0) {
      ro = R(q * itype);
      to = TR(q * itype);
    } else {
      const int64_t ipl = q * itype + r - 1;
      const double P = 1.0 - double(r) / double(LL);
      const double a1 = -P * (P - 1.0) * (P - 2.0) / 6.0, a2 = (P * P - 1.0) * (P - 2.0) * 0.5;
      const double a3 = -P * (P + 1.0) * (P - 2.0) * 0.5, a4 = P * (P * P - 1.0) / 6.0;
      ro = a1 * R(ipl - 1) + a2 * R(ipl) + a3 * R(ipl + 1) + a4 * R(ipl + 2);
      to = a1 * TR(ipl - 1) + a2 * TR(ipl) + a3 * TR(ipl + 1) + a4 * TR(ipl + 2);
    }
    rad = tr * ro + em;
    trn = tr * to;
    dr_do = -tr * ro + dem_do;
    rado = ro;
  }
  rad_out[f] = rad;
  tr_out[f] = trn;
  if (rows.mode == 1) {
    // the reference's layer rows (TDERIVup :6076-6110, QDERIVup :5900-5935)
    // from the quantities EMDT saves (:4500-4540); RADO is the radiance
    // entering the layer (the boundary emission under the first layer)
    const double bb = planck(vi, t.xkt, t.rk);
    const double bb_dif = xkta > 0. ? planck(vi, xkta, t.rka) - bb : 0.;
    const double betai = (bb + bb_dif) - bb;
    const double bbeff = bb + bb_dif * fi;
    const double bbd = planck_dt_ref(vi, t.xkt, bb);
    const double bbdt = xkta > 0. ? planck_dt_ref(vi, xkta, bb) : 0.;
    const double a = (bbeff + betai * fi - rado) * tr;
    for (int k = 0; k < rows.np; k++) {
      const double x = rows.dtau[k][f];
      double d;
      if (k + rows.k0 == 0) {
        const double optdpt = tr > 1.e-06 ? -log(tr) : x;
        const double dtaudt = x - optdpt;
        d = a * dtaudt + bbd * (1. - tr) + (1. - tr) * ((bbdt - bbd) * fi + betai * dfi * dtaudt);
      } else {
        d = x * (a + (1. - tr) * betai * dfi);
      }
      rows.d[k][f] = d;
    }
    return;
  }
  const double dbt = dem_db * planck_dt(vi, L.tave);
  for (int k = 0; k < rows.np; k++) {
    double d = clamped ? 0. : dr_do * rows.dtau[k][f];
    if (k + rows.k0 == 0) d += dbt;
    rows.d[k][f] = d;
  }
}

// Rows of lower layers carried through merge step k: row <- T_k * regrid(row)
// (RADNN's interpolation onto layer k's grid, then layer k's transmittance).
// Row r of the input lives at in + r*stride on grid k-1, output likewise on
// grid k.
__global__ void k_jac_prop(const LayerDev* Lp, const double* od, double dv_old, int64_t n_old,
                           const double* in, double* out, int64_t stride) {
  const LayerDev& L = *Lp;
  const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= L.npts) return;
  const double* x = in + (int64_t)blockIdx.y * stride;
  const double DV = L.dv;
  double tau = od[f];
  if (tau < -kODLO) tau = -kODLO;
  const double tr = exp(-tau);
  const long itype = (dv_old == DV) ? 0 : fint(DV / (dv_old - DV) + 0.5);
  auto X = [&](int64_t c) { return x[c < 0 ? 0 : (c >= n_old ? n_old - 1 : c)]; };
  double v;
  const int64_t LL = itype + 1;
  const int64_t q = f / LL, r = f % LL;
  if (itype == 0) {
    v = X(f);
  } else if (r == 0) {
    v = X(q * itype);
  } else {
    const int64_t ipl = q * itype + r - 1;
    const double P = 1.0 - double(r) / double(LL);
    const double a1 = -P * (P - 1.0) * (P - 2.0) / 6.0, a2 = (P * P - 1.0) * (P - 2.0) * 0.5;
    const double a3 = -P * (P + 1.0) * (P - 2.0) * 0.5, a4 = P * (P * P - 1.0) / 6.0;
    v = a1 * X(ipl - 1) + a2 * X(ipl) + a3 * X(ipl + 1) + a4 * X(ipl + 2);
  }
  out[(int64_t)blockIdx.y * stride + f] = tr * v;
}

// Top segment of layers a..L-1 sharing the top grid: each layer's row is
// carried to the top by the transmittance of the layers above it,
// accumulated downward point by point; rows of layers below a (already on
// the top grid, through layer a) take the product above layer a.
//   rows[(k*nlay + l)*n + i]  (in: d_p of layer l >= a, out: Jacobian row)
//   low[(k*a + j)*n + i]      (rows j < a carried through layer a)
__global__ void k_jac_top(const double* od, const int64_t* od_off, int nlay, int a, int np,
                          int64_t n, double* rows, const double* low) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double c = 1.;
  for (int m = nlay - 1; m >= a; m--) {
    for (int k = 0; k < np; k++) {
      double* r = rows + ((int64_t)k * nlay + m) * n + i;
      *r = *r * c;
    }
    if (m == a) {
      for (int k = 0; k < np; k++)
        for (int j = 0; j < a; j++)
          rows[((int64_t)k * nlay + j) * n + i] = low[((int64_t)k * a + j) * n + i] * c;
    }
    double tau = od[od_off[m] + i];
    if (tau < -kODLO) tau = -kODLO;
    c *= exp(-tau);
  }
}

// Means of each row of x (row r at x + r n) over the channels whose points
// are [cb[c], cb[c+1]): out[r nchan + c].  One CTA per (channel, row); the
// points of a channel are summed in a fixed order (thread stride, then a
// fixed reduction tree), so the result does not depend on timing.
__global__ void __launch_bounds__(256) k_chan_mean(const double* x, int64_t n, const int64_t* cb,
                                                   int64_t nchan, double* out) {
  __shared__ double red[8];
  const int64_t c = blockIdx.x, r = blockIdx.y;
  const int64_t a = cb[c], b = cb[c + 1];
  const double* xr = x + r * n;
  double s = 0.;
  for (int64_t i = a + threadIdx.x; i < b; i += blockDim.x) s += xr[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.;
    for (int k = 0; k < 8; k++) t += red[k];
    out[r * nchan + c] = b > a ? t / double(b - a) : 0.;
  }
}

// (tau(p+) - tau(p-)) / h, in place into plus
__global__ void k_jac_diff(double* plus, const double* minus, int64_t n, double rh) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) plus[i] = (plus[i] - minus[i]) * rh;
}

}  // namespace

template <int ADDERS, int DEC, int MINB>
void far_wing_attributes() {
  const cudaFuncAttribute c = cudaFuncAttributePreferredSharedMemoryCarveout;
  cudaFuncSetAttribute(k_far_wing<double, ADDERS, DEC, MINB>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, kFwSmem);
  cudaFuncSetAttribute(k_far_wing<float, ADDERS, DEC, MINB>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, fw_smem32(ADDERS));
  cudaFuncSetAttribute(k_far_wing<double, ADDERS, DEC, MINB>, c, cudaSharedmemCarveoutMaxShared);
  cudaFuncSetAttribute(k_far_wing<float, ADDERS, DEC, MINB>, c, cudaSharedmemCarveoutMaxShared);
}

template <typename T, int STAGE, int MINB>
void panel_carveout() {
  cudaFuncAttributes fa;
  int dev = 0, smem_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) !=
          cudaSuccess ||
      cudaFuncGetAttributes(&fa, k_panel_od<T, STAGE, MINB>) != cudaSuccess || smem_sm <= 0) {
    cudaGetLastError();
    return;
  }
  // MINB CTAs, each with its static shared memory and 1 KB the system keeps
  const double need = double(MINB) * double(fa.sharedSizeBytes + 1024);
  int pct = (int)std::ceil(100. * need / double(smem_sm));
  pct = pct < 1 ? 1 : (pct > 100 ? 100 : pct);
  cudaFuncSetAttribute(k_panel_od<T, STAGE, MINB>,
                       cudaFuncAttributePreferredSharedMemoryCarveout, pct);
}

void init_kernel_attributes() {
  // two R4 buffers per CTA (plus the FP32 accumulators of split precision);
  // the largest carveout lets three CTAs share an SM
  far_wing_attributes<160, 3, 3>();
  far_wing_attributes<128, 4, 3>();
  far_wing_attributes<192, 2, 3>();
  cudaFuncSetAttribute(k_near_walk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kNearWalkSmemMax);
  // the panel kernels read the shape tables (125 KB in FP64) through L1:
  // their shared-memory carveout is only what their CTAs per SM need, so
  // that the rest of the SM's 256 KB stays L1
  panel_carveout<double, 32, 4>();
  panel_carveout<double, 64, 4>();
  panel_carveout<double, 32, 5>();
  panel_carveout<float, 32, 4>();
  panel_carveout<float, 64, 4>();
  panel_carveout<float, 32, 5>();

}

void upload_voicon() {
  cudaMemcpyToSymbol(c_avrat, LBL_AVRAT, sizeof(LBL_AVRAT));
  cudaMemcpyToSymbol(c_cf1, LBL_CF1, sizeof(LBL_CF1));
  cudaMemcpyToSymbol(c_cf2, LBL_CF2, sizeof(LBL_CF2));
  cudaMemcpyToSymbol(c_cf3, LBL_CF3, sizeof(LBL_CF3));
  cudaMemcpyToSymbol(c_cgauss, LBL_CGAUSS, sizeof(LBL_CGAUSS));
  cudaMemcpyToSymbol(c_cer, LBL_CER, sizeof(LBL_CER));
  int iso[48] = {0};
  for (int m = 1; m <= 47; m++) iso[m] = LBL_ISO_MAX[m - 1];
  cudaMemcpyToSymbol(c_isomax, iso, sizeof(iso));
}

cudaError_t launch_far_scale(const Work& w, const DevLines& ln, int64_t max_far, cudaStream_t s) {
  if (max_far <= 0) return cudaSuccess;
  dim3 g((unsigned)((max_far + 255) / 256), (unsigned)w.nlay);
  k_far_scale<<<g, 256, 0, s>>>(w, ln);
  return cudaGetLastError();
}

cudaError_t launch_shrink(const Work& w, const int64_t* bs, const int64_t* blk_base,
                          int64_t nblk_total, cudaStream_t s) {
  // one warp per start block, then one warp per layer, then one warp per
  // segment; the plan runs also when no layer of the batch has far-wing
  // lines, since it sets every layer's shrunk-line, block and segment
  // counts (then 0) that the far-wing kernel reads
  if (nblk_total > 0)
    k_shr_count<<<(unsigned)((nblk_total + 3) / 4), 128, 0, s>>>(w, bs, blk_base, w.nlay);
  k_shr_plan<<<w.nlay, 32, 0, s>>>(w, blk_base);
  if (nblk_total > 0)
    k_shr_write<<<(unsigned)((nblk_total + 3) / 4), 128, 0, s>>>(w, bs, blk_base, w.nlay);
  return cudaGetLastError();
}

template <int ADDERS, int DEC, int MINB>
void launch_far_wing_v(const Work& w, int32_t nwin_total, const int32_t* win_order,
                       const int32_t* win_layer, int precision, cudaStream_t s) {
  constexpr int threads = ADDERS + 32 * DEC;
  if (precision == LBL_PREC_SPLIT)
    k_far_wing<float, ADDERS, DEC, MINB><<<nwin_total, threads, fw_smem32(ADDERS), s>>>(
        w, win_order, win_layer);
  else
    k_far_wing<double, ADDERS, DEC, MINB><<<nwin_total, threads, kFwSmem, s>>>(w, win_order,
                                                                                win_layer);
}

// Far-wing variants (adders, deciding warps, CTAs per SM): (160, 3, 3),
// (128, 4, 3), (192, 2, 3).
cudaError_t launch_far_wing(const Work& w, int32_t nwin_total, const int32_t* win_order,
                            const int32_t* win_layer, int precision, int variant,
                            cudaStream_t s) {
  if (nwin_total <= 0) return cudaSuccess;
  if (variant == 1)
    launch_far_wing_v<128, 4, 3>(w, nwin_total, win_order, win_layer, precision, s);
  else if (variant == 2)
    launch_far_wing_v<192, 2, 3>(w, nwin_total, win_order, win_layer, precision, s);
  else
    launch_far_wing_v<160, 3, 3>(w, nwin_total, win_order, win_layer, precision, s);
  return cudaGetLastError();
}

cudaError_t launch_near_lines(const Work& w, const DevLines& ln, int64_t max_near,
                              cudaStream_t s) {
  if (w.nlay > 65535) return cudaErrorInvalidValue;
  if (max_near > 0) {
    const dim3 g((unsigned)((max_near + 255) / 256), (unsigned)w.nlay);
    k_near_lines<<<g, 256, 0, s>>>(w, ln);
  }
  return cudaGetLastError();
}

cudaError_t launch_near_walk(const Work& w, const DevLines& ln, int64_t max_panel,
                             int64_t max_win, int64_t max_nblk, cudaStream_t s) {
  if (w.nlay > 65535) return cudaErrorInvalidValue;
  const size_t smem = near_walk_smem(max_panel, max_win);
  if (smem > kNearWalkSmemMax) return cudaErrorInvalidValue;
  k_near_walk<<<w.nlay, 32, smem, s>>>(w, ln);
  if (max_nblk > 0) k_near_out<<<dim3((unsigned)max_nblk, (unsigned)w.nlay), 256, 0, s>>>(w, ln);
  return cudaGetLastError();
}

cudaError_t launch_continuum(const Work& w, const DevMtckd& ck, double xself, double xfrgn,
                             double xrayl, double xco2c, double xo2cn, double xn2cn,
                             cudaStream_t s) {
  k_continuum<<<w.nlay, 256, 0, s>>>(w, ck, xself, xfrgn, xrayl, ContScale{xco2c, xo2cn, xn2cn});
  return cudaGetLastError();
}


cudaError_t launch_panel_segs(const Work& w, int64_t npanel_total, const int32_t* panel_layer,
                              const int64_t* panel_base, double* segs, int32_t* nseg,
                              cudaStream_t s) {
  if (npanel_total <= 0) return cudaSuccess;
  const unsigned nb = (unsigned)((npanel_total + 127) / 128);
  k_panel_segs<<<nb, 128, 0, s>>>(w, panel_layer, panel_base, npanel_total, segs, nseg);
  return cudaGetLastError();
}

cudaError_t launch_panel_ranges(const Work& w, int64_t npanel_total, const int32_t* panel_layer,
                                const int64_t* panel_base, int64_t* rng, cudaStream_t s) {
  if (npanel_total > 0)
    k_panel_ranges<<<(unsigned)((npanel_total + 127) / 128), 128, 0, s>>>(
        w, panel_layer, panel_base, npanel_total, rng);
  return cudaGetLastError();
}

// The panel kernel's variants: records staged per batch and the CTAs per SM
// the registers are bounded for: (32, 4), (64, 4), (32, 5).
int panel_stage_of(int variant) { return variant == 1 ? 64 : 32; }

template <typename T>
cudaError_t launch_panels_t(const Work& w, const DevShapes& sh, int64_t np,
                            const int32_t* panel_layer, const int64_t* panel_base,
                            const int64_t* rng, const double* segs, const int32_t* nseg,
                            int variant, cudaStream_t s) {
  const unsigned g = (unsigned)np;
  if (variant == 1)
    k_panel_od<T, 64, 4><<<g, kPanelThreads, 0, s>>>(w, sh, panel_layer, panel_base, rng, segs,
                                                      nseg);
  else if (variant == 2)
    k_panel_od<T, 32, 5><<<g, kPanelThreads, 0, s>>>(w, sh, panel_layer, panel_base, rng, segs,
                                                      nseg);
  else
    k_panel_od<T, 32, 4><<<g, kPanelThreads, 0, s>>>(w, sh, panel_layer, panel_base, rng, segs,
                                                      nseg);
  return cudaGetLastError();
}

cudaError_t launch_panels(const Work& w, const DevShapes& sh, int64_t npanel_total,
                          const int32_t* panel_layer, const int64_t* panel_base,
                          const int64_t* rng, const double* segs, const int32_t* nseg,
                          int precision, int variant, cudaStream_t s) {
  if (npanel_total <= 0) return cudaSuccess;
  if (npanel_total >= (int64_t(1) << 31)) return cudaErrorInvalidValue;
  if (precision == LBL_PREC_SPLIT)
    return launch_panels_t<float>(w, sh, npanel_total, panel_layer, panel_base, rng, segs, nseg,
                                  variant, s);
  return launch_panels_t<double>(w, sh, npanel_total, panel_layer, panel_base, rng, segs, nseg,
                                 variant, s);
}

cudaError_t launch_merge(const LayerDev* Ld, const double* vft_panel, const double* od,
                         int64_t npts, int first, double dv_old, int64_t n_old,
                         const double* rad_in, const double* tr_in, double* rad_out,
                         double* tr_out, double tbnd, double emis, int iemit, double tzu,
                         cudaStream_t s, int precision, int down, double tbnd_last,
                         double tzl_b, double refl) {
  if (npts >= (int64_t(1) << 31) || n_old >= (int64_t(1) << 31)) return cudaErrorInvalidValue;
  const unsigned nb = (unsigned)((npts + 255) / 256);
  if (precision == LBL_PREC_SPLIT)
    k_merge<float><<<nb, 256, 0, s>>>(Ld, vft_panel, od, first, dv_old, n_old, rad_in, tr_in,
                                      rad_out, tr_out, tbnd, emis, iemit, tzu, down, tbnd_last,
                                      tzl_b, refl);
  else
    k_merge<double><<<nb, 256, 0, s>>>(Ld, vft_panel, od, first, dv_old, n_old, rad_in, tr_in,
                                       rad_out, tr_out, tbnd, emis, iemit, tzu, down, tbnd_last,
                                      tzl_b, refl);
  return cudaGetLastError();
}

cudaError_t launch_merge_run(const MergeRun& m, const double* vft_panel, const double* od,
                             int64_t npts, double dv, const double* rad_in, const double* tr_in,
                             double* rad_out, double* tr_out, double tbnd, double emis, int iemit,
                             cudaStream_t s, int precision, int64_t f_lo, int64_t f_hi) {
  if (m.nl < 1 || m.nl > kMergeRunMax) return cudaErrorInvalidValue;
  if (npts >= (int64_t(1) << 31) || m.n_old < 0) return cudaErrorInvalidValue;
  if (f_hi < 0) f_hi = npts;
  if (f_lo < 0 || f_hi > npts || f_lo > f_hi) return cudaErrorInvalidValue;
  if (f_hi == f_lo) return cudaSuccess;
  const unsigned nb = (unsigned)((f_hi - f_lo + 255) / 256);
  const int32_t a = (int32_t)f_lo, b = (int32_t)f_hi;
  if (precision == LBL_PREC_SPLIT) {
    if (m.down)
      k_merge_run<float, true><<<nb, 256, 0, s>>>(m, vft_panel, od, a, b, dv, rad_in, tr_in,
                                                  rad_out, tr_out, tbnd, emis, iemit);
    else
      k_merge_run<float, false><<<nb, 256, 0, s>>>(m, vft_panel, od, a, b, dv, rad_in, tr_in,
                                                   rad_out, tr_out, tbnd, emis, iemit);
  } else if (m.tangent || m.refl > 0.) {
    k_merge_run<double, false><<<nb, 256, 0, s>>>(m, vft_panel, od, a, b, dv, rad_in, tr_in,
                                                  rad_out, tr_out, tbnd, emis, iemit);
  } else {
    constexpr int MK = kMergePointsPerThread;
    const int64_t g0 = (f_lo / (kMergeThreads * MK)) * (kMergeThreads * MK);
    const unsigned nb64 = (unsigned)((f_hi - g0 + kMergeThreads * MK - 1) / (kMergeThreads * MK));
    if (m.down)
      k_merge_run_f64<true, MK><<<nb64, kMergeThreads, 0, s>>>(
          m, vft_panel, od, a, b, dv, rad_in, tr_in, rad_out, tr_out, tbnd, emis, iemit);
    else
      k_merge_run_f64<false, MK><<<nb64, kMergeThreads, 0, s>>>(
          m, vft_panel, od, a, b, dv, rad_in, tr_in, rad_out, tr_out, tbnd, emis, iemit);
  }
  return cudaGetLastError();
}

}  // namespace lbl

namespace lbl {

cudaError_t launch_jac_layer(const LayerDev* Ld, const double* vft_panel, const double* od,
                             int64_t npts, int first, double dv_old, int64_t n_old,
                             const double* rad_in, const double* tr_in, double* rad_out,
                             double* tr_out, double tbnd, double emis, double tzu,
                             double* const* d, const double* const* dtau, int np,
                             int mode, int k0, cudaStream_t s) {
  if (np < 1 || np > kJacMaxPar) return cudaErrorInvalidValue;
  JacRows rows;
  rows.np = np;
  rows.mode = mode;
  rows.k0 = k0;
  for (int k = 0; k < kJacMaxPar; k++) {
    rows.d[k] = k < np ? d[k] : nullptr;
    rows.dtau[k] = k < np ? dtau[k] : nullptr;
  }
  k_jac_layer<<<(unsigned)((npts + 255) / 256), 256, 0, s>>>(
      Ld, vft_panel, od, first, dv_old, n_old, rad_in, tr_in, rad_out, tr_out, tbnd, emis, tzu,
      rows);
  return cudaGetLastError();
}

cudaError_t launch_jac_prop(const LayerDev* Ld, const double* od, int64_t npts, double dv_old,
                            int64_t n_old, const double* in, double* out, int64_t stride,
                            int nrows, cudaStream_t s) {
  if (nrows <= 0) return cudaSuccess;
  dim3 g((unsigned)((npts + 255) / 256), (unsigned)nrows);
  k_jac_prop<<<g, 256, 0, s>>>(Ld, od, dv_old, n_old, in, out, stride);
  return cudaGetLastError();
}

cudaError_t launch_jac_top(const double* od, const int64_t* od_off, int nlay, int a, int np,
                           int64_t n, double* rows, const double* low, cudaStream_t s) {
  k_jac_top<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(od, od_off, nlay, a, np, n, rows, low);
  return cudaGetLastError();
}

cudaError_t launch_chan_mean(const double* x, int64_t n, int nrows, const int64_t* cb,
                             int64_t nchan, double* out, cudaStream_t s) {
  if (nrows <= 0 || nchan <= 0) return cudaSuccess;
  if (nrows > 65535 || nchan >= (int64_t(1) << 31)) return cudaErrorInvalidValue;
  k_chan_mean<<<dim3((unsigned)nchan, (unsigned)nrows), 256, 0, s>>>(x, n, cb, nchan, out);
  return cudaGetLastError();
}

cudaError_t launch_jac_diff(double* plus, const double* minus, int64_t n, double rh,
                            cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_jac_diff<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(plus, minus, n, rh);
  return cudaGetLastError();
}

// ---- PNLINT (src/oprop.f90:1564-1806) ---------------------------------
// Output point II of a segment: FJJ = FJ1DIF + RATDV*(II-1), JJ = INT(FJJ)-2,
// JP = INT((FJJ-JJ)*100-199.5), value = A1(JP)*R1(JJ-1) + A2(JP)*R1(JJ) +
// A3(JP)*R1(JJ+1) + A4(JP)*R1(JJ+2) (label 30), every product and sum
// rounded separately and in that order.  R1(j) of input panel p is layer
// point g0+j-1; the first panel repeats R1(1) below j=1 (R1(-1)=R1(0)=R1(1))
// and the last repeats R1(NLIM) above NLIM (the two padded points).  Reads
// are HBM-bound gathers: each input point is read by about DV/DVOUT
// neighbouring threads of one CTA, so L1 serves the repeats.
__global__ void __launch_bounds__(256) k_pnlint(const PnlSeg* __restrict__ seg,
                                                const double* __restrict__ a,
                                                const double* __restrict__ od, int64_t n_in,
                                                double ratdv, double* __restrict__ out,
                                                int64_t n_out) {
  __shared__ double sa[4 * 101];
  for (int i = threadIdx.x; i < 4 * 101; i += blockDim.x) sa[i] = a[i];
  const PnlSeg S = seg[blockIdx.x];
  __syncthreads();
  const bool first = S.flags & 1, last = S.flags & 2;
  auto r1 = [&](long j) -> double {
    if (first && j < 1) j = 1;
    if (last && j > S.nlim) j = S.nlim;
    int64_t g = S.g0 + j - 1;
    g = g < 0 ? 0 : (g >= n_in ? n_in - 1 : g);
    return od[g];
  };
  for (int ii = S.ii_lo + (int)threadIdx.x; ii <= S.ii_hi; ii += blockDim.x) {
    const double fjj = __dadd_rn(S.fj1dif, __dmul_rn(ratdv, (double)(ii - 1)));
    const long jj = (long)fjj - 2;
    int jp = (int)__dsub_rn(__dmul_rn(__dsub_rn(fjj, (double)jj), 100.), 199.5);
    jp = jp < 0 ? 0 : (jp > 100 ? 100 : jp);
    double v = __dmul_rn(sa[jp], r1(jj - 1));
    v = __dadd_rn(v, __dmul_rn(sa[101 + jp], r1(jj)));
    v = __dadd_rn(v, __dmul_rn(sa[202 + jp], r1(jj + 1)));
    v = __dadd_rn(v, __dmul_rn(sa[303 + jp], r1(jj + 2)));
    const int64_t k = S.k0 + ii - 1;
    if (k < n_out) out[k] = v;
  }
}

cudaError_t launch_pnlint(const PnlSeg* seg, int64_t nseg, const double* a, const double* od,
                          int64_t n_in, double ratdv, double* out, int64_t n_out,
                          cudaStream_t s) {
  if (nseg <= 0) return cudaSuccess;
  if (nseg >= (int64_t(1) << 31) || n_in < 1) return cudaErrorInvalidValue;
  k_pnlint<<<(unsigned)nseg, 256, 0, s>>>(seg, a, od, n_in, ratdv, out, n_out);
  return cudaGetLastError();
}

// ---- SCANFN (src/postsub.f90:1276-1376 SHRKSC, :1516-1598 CONVSC) -------
__global__ void k_scan_compress(const double* __restrict__ spec, int64_t nc, int ir, int jabs,
                                double* __restrict__ sc) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nc) return;
  double sum = 0.;
  for (int j = 0; j < ir; j++) {
    double x = spec[k * ir + j];
    if (jabs) x = __dsub_rn(1., x);
    sum = __dadd_rn(sum, x);
  }
  sc[k] = __ddiv_rn(sum, (double)ir);
}

// Output point JF = 33 + j of the global grid: the inputs whose JMIN..JMAX
// holds JF (both bounds rise with the input index, found by bisection),
// summed in input order, each XNORM*S(I)*XF(|ZF|+1.5) with every product
// and sum rounded separately.
__device__ __forceinline__ double scan_zpeak(int64_t k, double ratio, double zint) {
  return __dadd_rn(__dmul_rn((double)(k - 1), ratio), zint);
}
__global__ void k_scan_gather(const double* __restrict__ sc, int64_t ilo, int64_t ihi,
                              double zint, double ratio, double zbound, double zslope,
                              double xnorm, const double* __restrict__ xf, int64_t nfmax,
                              double* __restrict__ out, int64_t n_out) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_out) return;
  const int64_t jf = 33 + j;
  auto jmax_of = [&](int64_t k) {
    return (int64_t)__dadd_rn(__dadd_rn(scan_zpeak(k, ratio, zint), zbound), 1.5);
  };
  auto jmin_of = [&](int64_t k) {
    return (int64_t)__dadd_rn(__dsub_rn(scan_zpeak(k, ratio, zint), zbound), 1.5);
  };
  // first k with JMAX >= JF
  int64_t lo = ilo, hi = ihi + 1;
  while (lo < hi) {
    const int64_t m = lo + (hi - lo) / 2;
    if (jmax_of(m) >= jf) hi = m;
    else lo = m + 1;
  }
  const int64_t k0 = lo;
  // last k with JMIN <= JF
  lo = ilo;
  hi = ihi + 1;
  while (lo < hi) {
    const int64_t m = lo + (hi - lo) / 2;
    if (jmin_of(m) <= jf) lo = m + 1;
    else hi = m;
  }
  const int64_t k1 = lo - 1;
  double acc = 0.;
  for (int64_t k = k0; k <= k1; k++) {
    const double s = sc[k - 1];
    if (s == 0.) continue;
    const double zpeak = scan_zpeak(k, ratio, zint);
    const double zf = __dmul_rn(__dsub_rn((double)(jf - 1), zpeak), zslope);
    int64_t it = (int64_t)__dadd_rn(fabs(zf), 1.5);
    it = it > nfmax ? nfmax : it;
    acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(xnorm, s), xf[it]));
  }
  out[j] = acc;
}

cudaError_t launch_scan(const double* spec, int64_t n, int ir, int jabs, double* sc, int64_t ilo,
                        int64_t ihi, double zint, double ratio, double zbound, double zslope,
                        double xnorm, const double* xf, int64_t nfmax, double* out,
                        int64_t n_out, cudaStream_t s) {
  const int64_t nc = n / ir;
  if (nc > 0)
    k_scan_compress<<<(unsigned)((nc + 255) / 256), 256, 0, s>>>(spec, nc, ir, jabs, sc);
  if (n_out > 0)
    k_scan_gather<<<(unsigned)((n_out + 255) / 256), 256, 0, s>>>(
        sc, ilo, ihi, zint, ratio, zbound, zslope, xnorm, xf, nfmax, out, n_out);
  return cudaGetLastError();
}

// CNVRCT (src/postsub.f90:1779-1985; mode 0), CNVVRC (:1986-2214; mode 5)
// and CNVVRL (:2216-2440; mode 6), one thread per box: the inner points
// weighted 1, the end points by the fraction of their interval inside the
// box, the weighted sum over the sum of the weights; the reference's order
// of operations, each rounded separately.  Box j: mode 0 centred at
// V1 + j DVO, half width HWHM; mode 5 centred there, from VCNT (1 - B^2/4)
// to VCNT (1 + B^2/4); mode 6 from VLFT = V1 + j DVO to VLFT (1 + B^2/2),
// B the field-of-view half angle in radians.
__device__ __forceinline__ void scan_box(int mode, double v1, double dvo, double hwhm, double bfov,
                                         int64_t j, double& vlft, double& vrgt) {
  const double v0 = __dadd_rn(v1, __dmul_rn((double)j, dvo));
  const double b2 = __dmul_rn(bfov, bfov);
  if (mode == 5) {
    const double q = __ddiv_rn(b2, 4.);
    vlft = __dmul_rn(v0, __dsub_rn(1., q));
    vrgt = __dmul_rn(v0, __dadd_rn(1., q));
  } else if (mode == 6) {
    vlft = v0;
    vrgt = __dmul_rn(v0, __dadd_rn(1., __ddiv_rn(b2, 2.)));
  } else {
    vlft = __dsub_rn(v0, hwhm);
    vrgt = __dadd_rn(v0, hwhm);
  }
}

__global__ void k_scan_rect(const double* __restrict__ spec, int64_t n, int jabs, int mode,
                            double v1, double dvo, double hwhm, double bfov, double v1i,
                            double dvi, double* __restrict__ out, int64_t n_out) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_out) return;
  auto S = [&](int64_t i) {  // 1-based
    const double x = spec[i - 1];
    return jabs ? __dsub_rn(1., x) : x;
  };
  double vlft, vrgt;
  scan_box(mode, v1, dvo, hwhm, bfov, j, vlft, vrgt);
  const double rl = __dadd_rn(__ddiv_rn(__dsub_rn(vlft, v1i), dvi), 1.);
  const double rr = __dadd_rn(__ddiv_rn(__dsub_rn(vrgt, v1i), dvi), 1.);
  int64_t il = (int64_t)__dadd_rn(rl, 0.5), ih = (int64_t)__dadd_rn(rr, 0.5);
  il = il < 1 ? 1 : il;
  ih = ih > n ? n : ih;
  const double half = __ddiv_rn(dvi, 2.);
  const double wgtl = __ddiv_rn(
      __dsub_rn(__dadd_rn(__dadd_rn(v1i, __dmul_rn((double)(il - 1), dvi)), half), vlft), dvi);
  const double wgtr = __ddiv_rn(
      __dsub_rn(vrgt, __dsub_rn(__dadd_rn(v1i, __dmul_rn((double)(ih - 1), dvi)), half)), dvi);
  double sum = 0.;
  for (int64_t i = il + 1; i <= ih - 1; i++) sum = __dadd_rn(sum, S(i));
  sum = __dadd_rn(sum, __dmul_rn(S(il), wgtl));
  sum = __dadd_rn(sum, __dmul_rn(S(ih), wgtr));
  const double rnj = __dadd_rn(__dadd_rn((double)(ih - il + 1 - 2), wgtl), wgtr);
  out[j] = __ddiv_rn(sum, rnj);
}

// SCNINT/INTERP (src/postsub.f90:2940-3215), one thread per chunk of output
// points: the 4-point cubic with weights tabulated at P = (IP-1)/200, P
// carried from point to point by adding DVO/DVI, as the reference does.
// T(i) of input panel k is spectrum point 2400 k + i - 5; below the first
// point T(4) = 2 T(5) - T(6) (and 0 further down), past the last point
// 2 S(n) - S(n-1) (and 0 further up), as INTERP sets them.
__global__ void k_scnint(const ScnChunkDev* __restrict__ chunks, int64_t nchunk,
                         const double* __restrict__ spec, int64_t n,
                         const double* __restrict__ coef, double vratio,
                         double* __restrict__ out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nchunk) return;
  const ScnChunkDev c = chunks[t];
  double* o = out + c.out0;
  if (c.zero) {
    for (int32_t j = 0; j < c.count; j++) o[j] = 0.;
    return;
  }
  auto T = [&](int64_t i) -> double {
    const int64_t g = 2400 * c.panel + i - 5;
    if (g < 0) return g == -1 ? __dsub_rn(__dmul_rn(2.0, spec[0]), spec[1]) : 0.;
    if (g >= n) return g == n ? __dsub_rn(__dmul_rn(2.0, spec[n - 1]), spec[n - 2]) : 0.;
    return spec[g];
  };
  int64_t I = c.i0;
  double P = c.p0;
  for (int32_t j = 0; j < c.count; j++) {
    int ip = (int)__dadd_rn(__dmul_rn(P, 201.), 1.00001);
    ip = ip < 0 ? 0 : (ip > 202 ? 202 : ip);
    double r = __dmul_rn(coef[ip], T(I - 1));
    r = __dadd_rn(r, __dmul_rn(coef[203 + ip], T(I)));
    r = __dadd_rn(r, __dmul_rn(coef[406 + ip], T(I + 1)));
    r = __dadd_rn(r, __dmul_rn(coef[609 + ip], T(I + 2)));
    o[j] = r;
    P = __dadd_rn(P, vratio);
    if (P >= 1.0) {
      I = (int64_t)__dadd_rn((double)I, P);
      P = __dsub_rn(P, (double)(int64_t)P);
    }
  }
}

cudaError_t launch_scnint(const ScnChunkDev* chunks, int64_t nchunk, const double* spec,
                          int64_t n, const double* coef, double vratio, double* out,
                          cudaStream_t s) {
  if (nchunk > 0)
    k_scnint<<<(unsigned)((nchunk + 127) / 128), 128, 0, s>>>(chunks, nchunk, spec, n, coef,
                                                              vratio, out);
  return cudaGetLastError();
}

cudaError_t launch_scan_rect(const double* spec, int64_t n, int jabs, int mode, double v1,
                             double dvo, double hwhm, double bfov, double v1i, double dvi,
                             double* out, int64_t n_out, cudaStream_t s) {
  if (n_out > 0)
    k_scan_rect<<<(unsigned)((n_out + 255) / 256), 256, 0, s>>>(spec, n, jabs, mode, v1, dvo,
                                                                 hwhm, bfov, v1i, dvi, out, n_out);
  return cudaGetLastError();
}

}  // namespace lbl
