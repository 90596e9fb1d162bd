// PARSEC wavefunction file (parsec.dat) reader and writer, host C++.
//
// The record sequence is the one shared/parsec_wfn.F90:80-320,663-700 reads,
// for a finite system (per = 0) with real orbitals and one spin channel:
//    1  datelabel                       character(len=26)
//    2  nspin, lcplx (0/1), per         3 x int32
//    3  step                            real(8)
//    4  ndim                            int32
//    5  shift                           3 x real(8)
//    6  nwedge, ntrans                  2 x int32
//    7  (skipped by the reader)
//    8  trans                           3 x 3 x ntrans real(8)
//    9, 10  (skipped)
//   11  chi                             ntrans x ntrans int32
//   12  gtable                          3 x nwedge int32
//   13  nstate                          int32
//   14  irep                            nstate int32
//   15  e0 (Ry)                         nstate real(8)
//   16  occ0                            nstate real(8)
//   17  (skipped)
//   18  rho                             nwedge real(8)
//   19-25  (skipped)
//   26  nn                              int32 (wavefunctions stored)
//   27  iord                            nn int32 (1-based state of each)
//   28..27+nn  one wavefunction each    nwedge real(8)
// Each record is Fortran sequential-unformatted: int32 byte count, payload,
// int32 byte count (gfortran's default 4-byte markers, native byte order).
// The skipped records are written empty.  Periodic, complex or
// spin-polarised files are reported as unsupported.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ngw_b200.h"

namespace ngw {
void set_error(const char *fmt, ...);
}

namespace {

struct Writer {
  FILE *f = nullptr;
  bool ok = true;
  void rec(const void *p, size_t n) {
    const uint32_t m = (uint32_t)n;
    ok = ok && fwrite(&m, 4, 1, f) == 1 && (n == 0 || fwrite(p, 1, n, f) == n) && fwrite(&m, 4, 1, f) == 1;
  }
};

struct Reader {
  FILE *f = nullptr;
  std::string err;
  // reads one record into out (resized), returns false on a malformed file
  bool rec(std::vector<char> &out) {
    uint32_t m1 = 0, m2 = 0;
    if (fread(&m1, 4, 1, f) != 1) {
      err = "unexpected end of file";
      return false;
    }
    out.resize(m1);
    if (m1 && fread(out.data(), 1, m1, f) != m1) {
      err = "truncated record";
      return false;
    }
    if (fread(&m2, 4, 1, f) != 1 || m2 != m1) {
      err = "record markers do not match";
      return false;
    }
    return true;
  }
  bool skip() {
    std::vector<char> tmp;
    return rec(tmp);
  }
  template <class T>
  bool get(T *dst, size_t count, const char *what) {
    std::vector<char> b;
    if (!rec(b)) return false;
    if (b.size() != count * sizeof(T)) {
      err = std::string("record '") + what + "' has " + std::to_string(b.size()) + " bytes, expected " +
            std::to_string(count * sizeof(T));
      return false;
    }
    if (count) std::memcpy(dst, b.data(), b.size());
    return true;
  }
};

int fail(const char *path, const std::string &why) {
  ngw::set_error("parsec.dat %s: %s", path, why.c_str());
  return NGW_ERR_ARG;
}

// Header records 1-16; fills h.  With the arrays null only the sizes are read.
int read_head(Reader &r, const char *path, ngw_parsec_header *h, double *trans, int *chi, int *gtable,
              int *irep, double *e0, double *occ) {
  std::vector<char> b;
  if (!r.rec(b)) return fail(path, r.err);
  std::memset(h->datelabel, 0, sizeof(h->datelabel));
  std::memcpy(h->datelabel, b.data(), std::min(b.size(), sizeof(h->datelabel) - 1));
  int t3[3];
  if (!r.get(t3, 3, "nspin, lcplx, per")) return fail(path, r.err);
  h->nspin = t3[0];
  h->lcplx = t3[1];
  h->per = t3[2];
  if (h->nspin != 1 || h->lcplx != 0 || h->per != 0)
    return fail(path, "only finite systems with real orbitals and one spin channel are supported (nspin " +
                          std::to_string(h->nspin) + ", complex " + std::to_string(h->lcplx) + ", per " +
                          std::to_string(h->per) + ")");
  if (!r.get(&h->step, 1, "step") || !r.get(&h->ndim, 1, "ndim") || !r.get(h->shift, 3, "shift"))
    return fail(path, r.err);
  int t2[2];
  if (!r.get(t2, 2, "nwedge, ntrans")) return fail(path, r.err);
  h->nwedge = t2[0];
  h->ntrans = t2[1];
  if (h->nwedge <= 0 || h->ntrans <= 0) return fail(path, "bad nwedge / ntrans");
  std::vector<double> tr((size_t)9 * h->ntrans);
  std::vector<int> ch((size_t)h->ntrans * h->ntrans);
  if (!r.skip() || !r.get(tr.data(), tr.size(), "trans") || !r.skip() || !r.skip() ||
      !r.get(ch.data(), ch.size(), "chi"))
    return fail(path, r.err);
  if (trans) std::memcpy(trans, tr.data(), tr.size() * 8);
  if (chi) std::memcpy(chi, ch.data(), ch.size() * 4);
  std::vector<int> gt((size_t)3 * h->nwedge);
  if (!r.get(gt.data(), gt.size(), "gtable")) return fail(path, r.err);
  if (gtable) std::memcpy(gtable, gt.data(), gt.size() * 4);
  if (!r.get(&h->nstate, 1, "nstate")) return fail(path, r.err);
  if (h->nstate <= 0) return fail(path, "no states");
  std::vector<int> ir(h->nstate);
  std::vector<double> e(h->nstate), oc(h->nstate);
  if (!r.get(ir.data(), ir.size(), "irep") || !r.get(e.data(), e.size(), "e0") ||
      !r.get(oc.data(), oc.size(), "occ0"))
    return fail(path, r.err);
  if (irep) std::memcpy(irep, ir.data(), ir.size() * 4);
  if (e0) std::memcpy(e0, e.data(), e.size() * 8);
  if (occ) std::memcpy(occ, oc.data(), oc.size() * 8);
  return NGW_OK;
}

}  // namespace

extern "C" int ngw_parsec_write(const char *path, const ngw_parsec_header *h, const int *gtable,
                                const double *rho, const int *irep, const double *e0, const double *occ,
                                const int *iord, const double *wfn, const double *trans, const int *chi) {
  if (!path || !h || !gtable || !rho || !irep || !e0 || !occ || !iord || !wfn || !trans || !chi ||
      h->nwedge <= 0 || h->ntrans <= 0 || h->nstate <= 0 || h->nwfn < 0) {
    ngw::set_error("ngw_parsec_write: bad arguments");
    return NGW_ERR_ARG;
  }
  if (h->nspin != 1 || h->lcplx != 0 || h->per != 0) {
    ngw::set_error("ngw_parsec_write: only finite systems with real orbitals and one spin channel");
    return NGW_ERR_ARG;
  }
  Writer w;
  w.f = fopen(path, "wb");
  if (!w.f) {
    ngw::set_error("ngw_parsec_write: cannot open %s", path);
    return NGW_ERR_ARG;
  }
  char label[26];
  std::memset(label, ' ', sizeof(label));
  std::memcpy(label, h->datelabel, std::min(strlen(h->datelabel), sizeof(label)));
  const int t3[3] = {h->nspin, h->lcplx, h->per};
  const int t2[2] = {h->nwedge, h->ntrans};
  w.rec(label, 26);
  w.rec(t3, 12);
  w.rec(&h->step, 8);
  w.rec(&h->ndim, 4);
  w.rec(h->shift, 24);
  w.rec(t2, 8);
  w.rec(nullptr, 0);
  w.rec(trans, (size_t)72 * h->ntrans);
  w.rec(nullptr, 0);
  w.rec(nullptr, 0);
  w.rec(chi, (size_t)4 * h->ntrans * h->ntrans);
  w.rec(gtable, (size_t)12 * h->nwedge);
  w.rec(&h->nstate, 4);
  w.rec(irep, (size_t)4 * h->nstate);
  w.rec(e0, (size_t)8 * h->nstate);
  w.rec(occ, (size_t)8 * h->nstate);
  w.rec(nullptr, 0);
  w.rec(rho, (size_t)8 * h->nwedge);
  for (int i = 0; i < 7; ++i) w.rec(nullptr, 0);
  w.rec(&h->nwfn, 4);
  w.rec(iord, (size_t)4 * h->nwfn);
  for (int k = 0; k < h->nwfn; ++k) w.rec(wfn + (size_t)k * h->nwedge, (size_t)8 * h->nwedge);
  const bool ok = w.ok && fclose(w.f) == 0;
  if (!ok) {
    ngw::set_error("ngw_parsec_write: write to %s failed", path);
    return NGW_ERR_ARG;
  }
  return NGW_OK;
}

extern "C" int ngw_parsec_read_header(const char *path, ngw_parsec_header *h) {
  if (!path || !h) {
    ngw::set_error("ngw_parsec_read_header: bad arguments");
    return NGW_ERR_ARG;
  }
  Reader r;
  r.f = fopen(path, "rb");
  if (!r.f) return fail(path, "cannot open");
  int rc = read_head(r, path, h, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
  if (rc == NGW_OK) {
    std::vector<char> b;
    bool ok = r.skip() && r.skip();   // 17 (skipped), 18 rho
    for (int i = 0; i < 7 && ok; ++i) ok = r.skip();
    if (!ok || !r.get(&h->nwfn, 1, "nn")) rc = fail(path, r.err);
  }
  fclose(r.f);
  return rc;
}

extern "C" int ngw_parsec_read(const char *path, ngw_parsec_header *h, int *gtable, double *rho, int *irep,
                               double *e0, double *occ, int *iord, double *wfn, double *trans, int *chi) {
  if (!path || !h || !gtable || !rho || !irep || !e0 || !occ || !iord || !wfn || !trans || !chi) {
    ngw::set_error("ngw_parsec_read: bad arguments");
    return NGW_ERR_ARG;
  }
  ngw_parsec_header want = *h;   // sizes the caller allocated for (from ngw_parsec_read_header)
  Reader r;
  r.f = fopen(path, "rb");
  if (!r.f) return fail(path, "cannot open");
  int rc = NGW_OK;
  do {
    ngw_parsec_header got;
    if ((rc = read_head(r, path, &got, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr)) != NGW_OK) break;
    if (got.nwedge != want.nwedge || got.ntrans != want.ntrans || got.nstate != want.nstate) {
      rc = fail(path, "sizes differ from the header the buffers were sized for");
      break;
    }
    rewind(r.f);
    if ((rc = read_head(r, path, h, trans, chi, gtable, irep, e0, occ)) != NGW_OK) break;
    if (!r.skip() || !r.get(rho, (size_t)h->nwedge, "rho")) {
      rc = fail(path, r.err);
      break;
    }
    bool ok = true;
    for (int i = 0; i < 7 && ok; ++i) ok = r.skip();
    int nn = 0;
    if (!ok || !r.get(&nn, 1, "nn")) {
      rc = fail(path, r.err);
      break;
    }
    if (nn != want.nwfn) {
      rc = fail(path, "number of stored wavefunctions differs from the header the buffers were sized for");
      break;
    }
    h->nwfn = nn;
    if (!r.get(iord, (size_t)nn, "iord")) {
      rc = fail(path, r.err);
      break;
    }
    for (int k = 0; k < nn && rc == NGW_OK; ++k)
      if (!r.get(wfn + (size_t)k * h->nwedge, (size_t)h->nwedge, "wavefunction")) rc = fail(path, r.err);
  } while (0);
  fclose(r.f);
  return rc;
}
