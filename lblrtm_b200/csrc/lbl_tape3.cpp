// lbl_tape3.cpp -- TAPE3 line-file reader (lbl_lines_load_tape3).
//
// TAPE3 is a Fortran unformatted sequential file (4-byte record markers,
// little-endian, the -frecord-marker=4 build of build/makefile.common):
//   record 1      file header; HLINID(7)(8:8) == '^' flags one extra record
//                 of negative-EPP bookkeeping (RDLIN, src/oprop.f90:745-751)
//   then pairs of records per panel:
//     INPUT_HEADER  VMIN, VMAX (REAL*8), NREC, NWDS (INTEGER*4)
//     INPUT_BLOCK   250 slots of VNU (REAL*8), SP, ALFA, EPP (REAL*4), MOL
//                   (INTEGER*4), HWHM, TMPALF, PSHIFT (REAL*4), IFLG
//                   (INTEGER*4), BRD_MOL_FLG_IN(7), BRD_MOL_DAT(21),
//                   SPEED_DEP (struct_types.f90:106-125)
// The shorter legacy block without the broadening fields, as the built-in
// test writer TESTMM produces (src/testmm.f90:206-227), is accepted too.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lblgpu.h"

namespace {

// One Fortran record: 1 read, 0 clean end of file (no bytes left), -1 a
// record cut short or with differing length markers.
int read_record(FILE* f, std::vector<char>& buf) {
  int32_t n1 = 0, n2 = 0;
  const size_t got = std::fread(&n1, 1, 4, f);
  if (got == 0 && std::feof(f)) return 0;
  if (got != 4) return -1;
  if (n1 < 0 || n1 > (1 << 28)) return -1;
  buf.resize(n1);
  if (n1 && std::fread(buf.data(), 1, n1, f) != (size_t)n1) return -1;
  if (std::fread(&n2, 4, 1, f) != 1) return -1;
  return n1 == n2 ? 1 : -1;
}

template <typename T>
T at(const std::vector<char>& b, size_t off) {
  T v;
  std::memcpy(&v, b.data() + off, sizeof(T));
  return v;
}

}  // namespace

extern "C" int lbl_tape3_parse(const char* path, std::vector<double>* vnu, std::vector<float>* sp,
                               std::vector<float>* alfa, std::vector<float>* epp,
                               std::vector<int32_t>* mol, std::vector<float>* hw,
                               std::vector<float>* tmp, std::vector<float>* psh,
                               std::vector<int32_t>* iflg, std::vector<int64_t>* bs,
                               std::string* err);

int lbl_tape3_parse(const char* path, std::vector<double>* vnu, std::vector<float>* sp,
                    std::vector<float>* alfa, std::vector<float>* epp, std::vector<int32_t>* mol,
                    std::vector<float>* hw, std::vector<float>* tmp, std::vector<float>* psh,
                    std::vector<int32_t>* iflg, std::vector<int64_t>* bs, std::string* err) {
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    *err = std::string("cannot open ") + path;
    return LBL_E_ARG;
  }
  std::vector<char> rec;
  if (read_record(f, rec) != 1 || rec.size() < 80) {
    std::fclose(f);
    *err = "TAPE3: missing file header record";
    return LBL_E_FORMAT;
  }
  if (rec[6 * 8 + 7] == '^') {
    if (read_record(f, rec) != 1) {
      std::fclose(f);
      *err = "TAPE3: missing negative-EPP record";
      return LBL_E_FORMAT;
    }
  }
  bs->clear();
  bs->push_back(0);
  const size_t NL = 250;
  for (;;) {
    const int hr = read_record(f, rec);
    if (hr == 0) break;  // end of file
    if (hr < 0) {
      std::fclose(f);
      *err = "TAPE3: truncated or malformed panel header record";
      return LBL_E_FORMAT;
    }
    if (rec.size() != 24) {
      std::fclose(f);
      *err = "TAPE3: panel header record is not 24 bytes";
      return LBL_E_FORMAT;
    }
    const int32_t nrec = at<int32_t>(rec, 16);
    std::vector<char> blk;
    if (read_record(f, blk) != 1) {
      std::fclose(f);
      *err = "TAPE3: truncated panel";
      return LBL_E_FORMAT;
    }
    if (nrec < 0 || nrec > 250) {
      std::fclose(f);
      *err = "RDLIN; NREC GT LIMIN";
      return LBL_E_NREC;
    }
    const bool full = blk.size() >= NL * 156;
    const bool legacy = blk.size() >= NL * 40 && !full;
    if (!full && !legacy) {
      std::fclose(f);
      *err = "TAPE3: panel data record has an unknown size";
      return LBL_E_FORMAT;
    }
    // field offsets of the 250-slot arrays
    const size_t o_vnu = 0, o_sp = NL * 8, o_alfa = o_sp + NL * 4, o_epp = o_alfa + NL * 4,
                 o_mol = o_epp + NL * 4, o_hw = o_mol + NL * 4, o_tmp = o_hw + NL * 4,
                 o_psh = o_tmp + NL * 4, o_iflg = o_psh + NL * 4;
    for (int32_t k = 0; k < nrec; k++) {
      vnu->push_back(at<double>(blk, o_vnu + 8 * k));
      sp->push_back(at<float>(blk, o_sp + 4 * k));
      alfa->push_back(at<float>(blk, o_alfa + 4 * k));
      epp->push_back(at<float>(blk, o_epp + 4 * k));
      mol->push_back(at<int32_t>(blk, o_mol + 4 * k));
      hw->push_back(at<float>(blk, o_hw + 4 * k));
      tmp->push_back(at<float>(blk, o_tmp + 4 * k));
      psh->push_back(at<float>(blk, o_psh + 4 * k));
      iflg->push_back(at<int32_t>(blk, o_iflg + 4 * k));
    }
    if (nrec > 0) bs->push_back((int64_t)vnu->size());
  }
  std::fclose(f);
  return LBL_OK;
}
