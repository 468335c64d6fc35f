// Trajectory readers without MDAnalysis: GROMACS TRR and XTC, CHARMM/NAMD DCD.
//
// The reference reads frames through MDAnalysis (pycusaxs/topology.py:52-75,
// 621-737) and converts GROMACS nanometres to Angstrom on the way; these
// readers do the same conversion and return positions (natoms x 3, Angstrom)
// and the box as three row vectors (Angstrom), the layout the SAXS path takes.
//
// TRR: a sequence of XDR (big-endian) frames, each a header
//   magic 1993, version string "GMX_trn_file", the byte sizes of the optional
//   blocks (ir, e, box, vir, pres, top, sym, x, v, f), natoms, step, nre,
//   time and lambda (float or double, following the block sizes)
// followed by the blocks present (box 3x3, virial, pressure, x, v, f).
// DCD: Fortran unformatted records (length markers around each record):
//   84-byte header ("CORD", 20 control ints: frame count, unit-cell flag,
//   ...), a title record, the atom count, then per frame an optional unit-cell
//   record of six doubles (a, gamma, b, beta, alpha, c; angles in degrees or
//   as cosines) and three records of natoms floats (x, y, z).
// XTC: XDR frames of magic 1995, natoms, step, time (float), the box (9 floats,
//   nm), natoms again, then the coordinates: 3*natoms plain floats for at most
//   9 atoms, else GROMACS's compressed form (see xtc_decode below).
// All are indexed once at open (frame byte offsets) for random access; reads
// use pread, so concurrent saxs_traj_read calls on one handle are safe.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include "pycusaxs_b200.h"
#include "scratch_forward.h"

namespace {

int terr(int code, const std::string &msg) { return saxs::record_error(code, msg.c_str()); }

uint32_t be32(const unsigned char *p) {
  return (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) | (uint32_t(p[2]) << 8) | uint32_t(p[3]);
}

uint32_t le32(const unsigned char *p) {
  return (uint32_t(p[3]) << 24) | (uint32_t(p[2]) << 16) | (uint32_t(p[1]) << 8) | uint32_t(p[0]);
}

float f32_from(uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

double f64_from(uint64_t u) {
  double d;
  std::memcpy(&d, &u, 8);
  return d;
}

// Box rows from edge lengths and angles (degrees): a along x, b in the xy plane.
void box_from_lengths(double a, double b, double c, double alpha, double beta, double gamma, float out[9]) {
  const double d2r = M_PI / 180.0;
  const double ca = std::cos(alpha * d2r), cb = std::cos(beta * d2r), cg = std::cos(gamma * d2r);
  const double sg = std::sin(gamma * d2r);
  const double cx = c * cb;
  const double cy = c * (ca - cb * cg) / sg;
  const double cz2 = c * c - cx * cx - cy * cy;
  const double cz = cz2 > 0.0 ? std::sqrt(cz2) : 0.0;
  const double rows[9] = {a, 0.0, 0.0, b * cg, b * sg, 0.0, cx, cy, cz};
  for (int i = 0; i < 9; ++i) out[i] = static_cast<float>(std::fabs(rows[i]) < 1e-9 ? 0.0 : rows[i]);
}

}  // namespace

struct SaxsTraj {
  int fd = -1;
  int format = 0;  // SAXS_TRAJ_TRR, SAXS_TRAJ_DCD or SAXS_TRAJ_XTC
  int natoms = 0;
  std::vector<int64_t> offsets;  // byte offset of every frame
  // TRR
  std::vector<int> trr_double;  // per frame: reals are doubles
  // DCD
  bool dcd_le = true;
  bool dcd_cell = false;
  double dcd_dt = 0.0;
};

namespace {

bool read_at(const SaxsTraj *t, int64_t off, void *dst, size_t n) {
  unsigned char *p = static_cast<unsigned char *>(dst);
  while (n > 0) {
    const ssize_t r = ::pread(t->fd, p, n, static_cast<off_t>(off));
    if (r <= 0) return false;
    p += r;
    off += r;
    n -= static_cast<size_t>(r);
  }
  return true;
}

struct TrrHeader {
  int sizes[10];  // ir, e, box, vir, pres, top, sym, x, v, f
  int natoms, step, nre;
  bool dbl;
  double time;
  int64_t header_bytes;
};

int trr_header(const SaxsTraj *t, int64_t off, TrrHeader *h) {
  unsigned char b[200];
  if (!read_at(t, off, b, 12)) return 1;  // end of file
  if (be32(b) != 1993u) return terr(SAXS_E_INVALID, "TRR: bad magic at byte " + std::to_string(off));
  const uint32_t slen = be32(b + 8);  // XDR string length of the version string
  const int64_t spad = (slen + 3) / 4 * 4;
  if (slen > 64) return terr(SAXS_E_INVALID, "TRR: implausible version string length");
  const int64_t p = 12 + spad;
  if (!read_at(t, off + p, b, 13 * 4)) return terr(SAXS_E_INVALID, "TRR: truncated header");
  for (int i = 0; i < 10; ++i) h->sizes[i] = static_cast<int>(be32(b + 4 * i));
  h->natoms = static_cast<int>(be32(b + 40));
  h->step = static_cast<int>(be32(b + 44));
  h->nre = static_cast<int>(be32(b + 48));
  if (h->natoms <= 0) return terr(SAXS_E_INVALID, "TRR: frame without atoms");
  int real = 0;
  if (h->sizes[2]) real = h->sizes[2] / 9;
  else if (h->sizes[7]) real = h->sizes[7] / (3 * h->natoms);
  else if (h->sizes[8]) real = h->sizes[8] / (3 * h->natoms);
  else if (h->sizes[9]) real = h->sizes[9] / (3 * h->natoms);
  if (real != 4 && real != 8) return terr(SAXS_E_INVALID, "TRR: cannot tell the precision of a frame");
  h->dbl = real == 8;
  unsigned char tb[16];
  if (!read_at(t, off + p + 52, tb, 2 * real)) return terr(SAXS_E_INVALID, "TRR: truncated header");
  if (h->dbl)
    h->time = f64_from((uint64_t(be32(tb)) << 32) | be32(tb + 4));
  else
    h->time = f32_from(be32(tb));
  h->header_bytes = p + 52 + 2 * real;
  return 0;
}

int open_trr(SaxsTraj *t) {
  int64_t off = 0;
  TrrHeader h;
  for (;;) {
    const int rc = trr_header(t, off, &h);
    if (rc == 1) break;
    if (rc) return rc;
    if (t->natoms == 0) t->natoms = h.natoms;
    if (h.natoms != t->natoms) return terr(SAXS_E_INVALID, "TRR: the atom count changes between frames");
    if (h.sizes[7] == 0) return terr(SAXS_E_INVALID, "TRR: a frame without coordinates");
    t->offsets.push_back(off);
    t->trr_double.push_back(h.dbl ? 1 : 0);
    int64_t body = 0;
    for (int i = 0; i < 10; ++i) body += h.sizes[i];
    off += h.header_bytes + body;
  }
  if (t->offsets.empty()) return terr(SAXS_E_INVALID, "TRR: no frames");
  return SAXS_OK;
}

int read_trr(const SaxsTraj *t, int64_t frame, float *xyz, float box[9], double *time) {
  TrrHeader h;
  const int rc = trr_header(t, t->offsets[frame], &h);
  if (rc) return rc == 1 ? terr(SAXS_E_INVALID, "TRR: frame vanished") : rc;
  int64_t p = t->offsets[frame] + h.header_bytes + h.sizes[0] + h.sizes[1];
  const int n3 = 3 * h.natoms;
  double bx[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (h.dbl) {
    std::vector<uint64_t> raw(static_cast<size_t>(std::max(n3, 9)));
    if (h.sizes[2]) {
      if (!read_at(t, p, raw.data(), 72)) return terr(SAXS_E_INVALID, "TRR: truncated box");
      for (int i = 0; i < 9; ++i) bx[i] = f64_from(__builtin_bswap64(raw[i]));
    }
    p += h.sizes[2] + h.sizes[3] + h.sizes[4] + h.sizes[5] + h.sizes[6];
    if (!read_at(t, p, raw.data(), static_cast<size_t>(n3) * 8))
      return terr(SAXS_E_INVALID, "TRR: truncated coordinates");
    for (int i = 0; i < n3; ++i) xyz[i] = static_cast<float>(10.0 * f64_from(__builtin_bswap64(raw[i])));
  } else {
    uint32_t rb[9];
    if (h.sizes[2]) {
      if (!read_at(t, p, rb, 36)) return terr(SAXS_E_INVALID, "TRR: truncated box");
      for (int i = 0; i < 9; ++i) bx[i] = f32_from(__builtin_bswap32(rb[i]));
    }
    p += h.sizes[2] + h.sizes[3] + h.sizes[4] + h.sizes[5] + h.sizes[6];
    // read straight into the output, then swap bytes and scale in place
    uint32_t *raw = reinterpret_cast<uint32_t *>(xyz);
    if (!read_at(t, p, raw, static_cast<size_t>(n3) * 4))
      return terr(SAXS_E_INVALID, "TRR: truncated coordinates");
    for (int i = 0; i < n3; ++i) xyz[i] = static_cast<float>(10.0 * f32_from(__builtin_bswap32(raw[i])));
  }
  // nanometres -> Angstrom
  for (int i = 0; i < 9; ++i) box[i] = static_cast<float>(10.0 * bx[i]);
  if (time) *time = h.time;
  return SAXS_OK;
}

int open_dcd(SaxsTraj *t) {
  unsigned char b[96];
  if (!read_at(t, 0, b, 92)) return terr(SAXS_E_INVALID, "DCD: file too short");
  if (le32(b) == 84u) t->dcd_le = true;
  else if (be32(b) == 84u) t->dcd_le = false;
  else return terr(SAXS_E_INVALID, "DCD: first record is not the 84-byte header");
  auto rd = [&](const unsigned char *p) { return t->dcd_le ? le32(p) : be32(p); };
  if (std::memcmp(b + 4, "CORD", 4) != 0) return terr(SAXS_E_INVALID, "DCD: missing CORD tag");
  const unsigned char *ic = b + 8;  // 20 control ints
  const int nset = static_cast<int>(rd(ic));
  const int namnf = static_cast<int>(rd(ic + 4 * 8));
  t->dcd_dt = f32_from(rd(ic + 4 * 9));
  const int charmm = static_cast<int>(rd(ic + 4 * 19));
  t->dcd_cell = charmm != 0 && rd(ic + 4 * 10) != 0;
  if (namnf != 0) return terr(SAXS_E_INVALID, "DCD: fixed atoms are not supported");
  if (rd(b + 88) != 84u) return terr(SAXS_E_INVALID, "DCD: bad header record end");
  int64_t off = 92;
  unsigned char m[8];
  if (!read_at(t, off, m, 4)) return terr(SAXS_E_INVALID, "DCD: missing title record");
  const uint32_t tlen = rd(m);
  off += 4 + tlen + 4;
  if (!read_at(t, off, m, 8) || rd(m) != 4u) return terr(SAXS_E_INVALID, "DCD: missing atom-count record");
  t->natoms = static_cast<int>(rd(m + 4));
  off += 12;
  if (t->natoms <= 0) return terr(SAXS_E_INVALID, "DCD: no atoms");
  const int64_t frame_bytes = (t->dcd_cell ? 56 : 0) + 3 * (8 + 4 * static_cast<int64_t>(t->natoms));
  struct stat sb;
  if (fstat(t->fd, &sb) != 0) return terr(SAXS_E_INVALID, "DCD: cannot stat the file");
  const int64_t size = static_cast<int64_t>(sb.st_size);
  const int64_t avail = (size - off) / frame_bytes;
  const int64_t n = nset > 0 ? std::min<int64_t>(nset, avail) : avail;
  for (int64_t k = 0; k < n; ++k) t->offsets.push_back(off + k * frame_bytes);
  if (t->offsets.empty()) return terr(SAXS_E_INVALID, "DCD: no frames");
  return SAXS_OK;
}

int read_dcd(const SaxsTraj *t, int64_t frame, float *xyz, float box[9], double *time) {
  auto rd = [&](const unsigned char *p) { return t->dcd_le ? le32(p) : be32(p); };
  int64_t p = t->offsets[frame];
  const int n = t->natoms;
  if (t->dcd_cell) {
    unsigned char c[56];
    if (!read_at(t, p, c, 56) || rd(c) != 48u) return terr(SAXS_E_INVALID, "DCD: bad unit-cell record");
    double u[6];
    for (int i = 0; i < 6; ++i) {
      const unsigned char *q = c + 4 + 8 * i;
      const uint64_t lo = rd(q), hi = rd(q + 4);
      u[i] = t->dcd_le ? f64_from((hi << 32) | lo) : f64_from((lo << 32) | hi);
    }
    // record order a, gamma, b, beta, alpha, c; angles may be stored as cosines
    double al = u[4], be = u[3], ga = u[1];
    if (std::fabs(al) <= 1.0 && std::fabs(be) <= 1.0 && std::fabs(ga) <= 1.0) {
      al = std::acos(al) * 180.0 / M_PI;
      be = std::acos(be) * 180.0 / M_PI;
      ga = std::acos(ga) * 180.0 / M_PI;
    }
    box_from_lengths(u[0], u[2], u[5], al, be, ga, box);
    p += 56;
  } else {
    for (int i = 0; i < 9; ++i) box[i] = 0.0f;
  }
  std::vector<unsigned char> buf(static_cast<size_t>(4) * n + 8);
  for (int d = 0; d < 3; ++d) {
    if (!read_at(t, p, buf.data(), buf.size()) || rd(buf.data()) != 4u * n)
      return terr(SAXS_E_INVALID, "DCD: bad coordinate record");
    for (int i = 0; i < n; ++i) xyz[3 * i + d] = f32_from(rd(buf.data() + 4 + 4 * i));
    p += 4 * static_cast<int64_t>(n) + 8;
  }
  if (time) *time = t->dcd_dt * static_cast<double>(frame);
  return SAXS_OK;
}

// ---- XTC ----------------------------------------------------------------------
//
// The compressed coordinates of an XTC frame, as GROMACS's xdr3dfcoord writes
// them (the published format; this is an independent implementation):
//   float precision p; int minint[3], maxint[3]; int smallidx; int nbytes;
//   nbytes of a bit stream (XDR opaque, padded to 4 bytes).
// Coordinates are integers round(x * p).  The stream holds groups:
//   * one "large" atom: its three integers minus minint, either as one
//     mixed-radix number of bit_length(size0 * size1 * size2) bits (size_d =
//     maxint_d - minint_d + 1), or, when a size exceeds 2^24 - 1, as three
//     numbers of bit_length(size_d) bits each;
//   * one flag bit; when set, 5 bits v give the run length run = v - v % 3
//     (three times the number of small atoms that follow) and a change of the
//     small-delta precision, v % 3 - 1 in {-1, 0, +1}; when clear, the previous
//     run length is kept and the precision stays;
//   * run / 3 "small" atoms: three integers in [0, m) with m = kMagic[smallidx],
//     as one mixed-radix number of smallidx bits, each the difference to the
//     previous atom plus m / 2.  The first small atom of a group and the large
//     atom are written in swapped order (the small one comes first in the
//     frame), which compresses water well;
//   * then smallidx changes by the group's precision change.
// Numbers are read most-significant bit first; a mixed-radix number of k bits
// arrives as bytes from the least significant up, the last one holding the
// remaining k - 8 * floor((k - 1) / 8) bits.
//
// kMagic[i] ~ 2^(i/3): the table of small-delta ranges of the format (it has to
// be the writer's, value for value, to read its files).
constexpr int kXtcFirstIdx = 9;
constexpr int kMagic[] = {
    0,       0,       0,       0,       0,       0,       0,       0,       0,       8,       10,
    12,      16,      20,      25,      32,      40,      50,      64,      80,      101,     128,
    161,     203,     256,     322,     406,     512,     645,     812,     1024,    1290,    1625,
    2048,    2580,    3250,    4096,    5060,    6501,    8192,    10321,   13003,   16384,   20642,
    26007,   32768,   41285,   52015,   65536,   82570,   104031,  131072,  165140,  208063,  262144,
    330280,  416127,  524287,  660561,  832255,  1048576, 1321122, 1664510, 2097152, 2642245, 3329021,
    4194304, 5284491, 6658042, 8388607, 10568983, 13316085, 16777216};
constexpr int kXtcLastIdx = static_cast<int>(sizeof(kMagic) / sizeof(kMagic[0])) - 1;

// Most-significant-bit-first reader over the frame's bytes.
struct BitStream {
  const unsigned char *p;
  size_t nbits;
  size_t pos = 0;
  bool overrun = false;
  uint32_t take(int n) {  // n <= 32
    if (pos + static_cast<size_t>(n) > nbits) {
      overrun = true;
      return 0;
    }
    uint32_t v = 0;
    for (int k = 0; k < n;) {
      const int off = static_cast<int>(pos & 7);
      const int m = std::min(8 - off, n - k);
      v = (v << m) | ((p[pos >> 3] >> (8 - off - m)) & ((1u << m) - 1u));
      k += m;
      pos += m;
    }
    return v;
  }
  // a k-bit mixed-radix number (k <= 96) split into three digits of the radices r
  void triple(int k, const uint32_t r[3], int out[3]) {
    unsigned __int128 n = 0;
    int shift = 0;
    while (k > 8) {
      n |= static_cast<unsigned __int128>(take(8)) << shift;
      shift += 8;
      k -= 8;
    }
    n |= static_cast<unsigned __int128>(take(k)) << shift;
    out[2] = static_cast<int>(n % r[2]);
    n /= r[2];
    out[1] = static_cast<int>(n % r[1]);
    n /= r[1];
    out[0] = static_cast<int>(n > 0xFFFFFFFFu ? 0xFFFFFFFFu : static_cast<uint32_t>(n));
  }
};

int bit_length(unsigned __int128 v) {
  int b = 0;
  while (v) {
    ++b;
    v >>= 1;
  }
  return b;
}

int xtc_header(const SaxsTraj *t, int64_t off, int *natoms, int64_t *frame_bytes) {
  unsigned char b[92];
  if (!read_at(t, off, b, 4)) return 1;  // end of file
  if (be32(b) != 1995u) return terr(SAXS_E_INVALID, "XTC: bad magic at byte " + std::to_string(off));
  if (!read_at(t, off, b, 56)) return terr(SAXS_E_INVALID, "XTC: truncated frame header");
  const int n = static_cast<int>(be32(b + 4));
  if (n <= 0 || static_cast<int>(be32(b + 52)) != n) return terr(SAXS_E_INVALID, "XTC: bad atom count");
  *natoms = n;
  if (n <= 9) {
    *frame_bytes = 56 + 12 * static_cast<int64_t>(n);
    return 0;
  }
  if (!read_at(t, off + 56, b, 36)) return terr(SAXS_E_INVALID, "XTC: truncated coordinate header");
  const int64_t nbytes = be32(b + 32);
  *frame_bytes = 56 + 36 + (nbytes + 3) / 4 * 4;
  return 0;
}

int open_xtc(SaxsTraj *t) {
  struct stat sb;
  if (fstat(t->fd, &sb) != 0) return terr(SAXS_E_INVALID, "XTC: cannot stat the file");
  int64_t off = 0;
  for (;;) {
    int n = 0;
    int64_t fb = 0;
    const int rc = xtc_header(t, off, &n, &fb);
    if (rc == 1) break;
    if (rc) return rc;
    if (off + fb > static_cast<int64_t>(sb.st_size)) return terr(SAXS_E_INVALID, "XTC: truncated last frame");
    if (t->natoms == 0) t->natoms = n;
    if (n != t->natoms) return terr(SAXS_E_INVALID, "XTC: the atom count changes between frames");
    t->offsets.push_back(off);
    off += fb;
  }
  if (t->offsets.empty()) return terr(SAXS_E_INVALID, "XTC: no frames");
  return SAXS_OK;
}

// Decode one frame's coordinates into xyz (nm); returns an error for a stream
// that does not fit its own header (never reads or writes out of bounds).
int xtc_decode(const unsigned char *hdr, const unsigned char *data, size_t nbytes, int natoms, float *xyz) {
  const float precision = f32_from(be32(hdr));
  if (!(precision > 0.0f)) return terr(SAXS_E_INVALID, "XTC: non-positive precision");
  const float inv = static_cast<float>(1.0 / static_cast<double>(precision));
  int minint[3], maxint[3];
  for (int d = 0; d < 3; ++d) {
    minint[d] = static_cast<int>(be32(hdr + 4 + 4 * d));
    maxint[d] = static_cast<int>(be32(hdr + 16 + 4 * d));
  }
  int smallidx = static_cast<int>(be32(hdr + 28));
  uint32_t size[3];
  bool large = false;
  for (int d = 0; d < 3; ++d) {
    const int64_t sz = static_cast<int64_t>(maxint[d]) - minint[d] + 1;
    if (sz <= 0 || sz > 0xFFFFFFFFll) return terr(SAXS_E_INVALID, "XTC: bad coordinate range");
    size[d] = static_cast<uint32_t>(sz);
    large |= sz > 0xFFFFFF;
  }
  int bits3 = 0, bits1[3] = {0, 0, 0};
  if (large) {
    for (int d = 0; d < 3; ++d) bits1[d] = bit_length(size[d]);
  } else {
    bits3 = bit_length(static_cast<unsigned __int128>(size[0]) * size[1] * size[2]);
  }
  if (smallidx < kXtcFirstIdx || smallidx > kXtcLastIdx) return terr(SAXS_E_INVALID, "XTC: bad small-delta index");
  BitStream bs{data, 8 * nbytes};
  int run = 0, i = 0;
  float *out = xyz;
  auto emit = [&](const int c[3]) {
    for (int d = 0; d < 3; ++d) *out++ = static_cast<float>(c[d]) * inv;
  };
  while (i < natoms) {
    int big[3];
    if (large) {
      for (int d = 0; d < 3; ++d) big[d] = static_cast<int>(bs.take(bits1[d]));
    } else {
      bs.triple(bits3, size, big);
    }
    for (int d = 0; d < 3; ++d) big[d] += minint[d];
    ++i;
    int change = 0;
    if (bs.take(1)) {
      const int v = static_cast<int>(bs.take(5));
      change = v % 3 - 1;
      run = v - v % 3;
    }
    if (bs.overrun) return terr(SAXS_E_INVALID, "XTC: compressed coordinates end early");
    if (run > 0) {
      if (i + run / 3 > natoms) return terr(SAXS_E_INVALID, "XTC: a run passes the last atom");
      const uint32_t m = static_cast<uint32_t>(kMagic[smallidx]);
      const uint32_t msz[3] = {m, m, m};
      const int half = kMagic[smallidx] / 2;
      int prev[3] = {big[0], big[1], big[2]};
      for (int k = 0; k < run; k += 3) {
        int c[3];
        bs.triple(smallidx, msz, c);
        for (int d = 0; d < 3; ++d) c[d] += prev[d] - half;
        ++i;
        if (k == 0) {
          emit(c);    // the first small atom precedes the large one
          emit(big);
        } else {
          emit(c);
        }
        for (int d = 0; d < 3; ++d) prev[d] = c[d];
      }
    } else {
      emit(big);
    }
    smallidx += change;
    if (smallidx < kXtcFirstIdx || smallidx > kXtcLastIdx) return terr(SAXS_E_INVALID, "XTC: bad small-delta index");
    if (bs.overrun) return terr(SAXS_E_INVALID, "XTC: compressed coordinates end early");
  }
  return SAXS_OK;
}

int read_xtc(const SaxsTraj *t, int64_t frame, float *xyz, float box[9], double *time) {
  const int64_t off = t->offsets[frame];
  unsigned char h[92];
  if (!read_at(t, off, h, 56)) return terr(SAXS_E_INVALID, "XTC: frame vanished");
  const int n = t->natoms;
  for (int i = 0; i < 9; ++i) box[i] = f32_from(be32(h + 16 + 4 * i)) * 10.0f;  // nm -> Angstrom
  if (time) *time = f32_from(be32(h + 12));
  if (n <= 9) {
    unsigned char b[108];
    if (!read_at(t, off + 56, b, 12 * static_cast<size_t>(n))) return terr(SAXS_E_INVALID, "XTC: truncated frame");
    for (int i = 0; i < 3 * n; ++i) xyz[i] = f32_from(be32(b + 4 * i)) * 10.0f;
    return SAXS_OK;
  }
  if (!read_at(t, off + 56, h + 56, 36)) return terr(SAXS_E_INVALID, "XTC: truncated frame");
  const size_t nbytes = be32(h + 88);
  std::vector<unsigned char> data(nbytes + 1);
  if (!read_at(t, off + 92, data.data(), nbytes)) return terr(SAXS_E_INVALID, "XTC: truncated frame");
  if (int rc = xtc_decode(h + 56, data.data(), nbytes, n, xyz)) return rc;
  for (int i = 0; i < 3 * n; ++i) xyz[i] *= 10.0f;  // nm -> Angstrom
  return SAXS_OK;
}

}  // namespace

extern "C" {

int saxs_traj_open(const char *path, int format, SaxsTraj **out) {
  if (!path || !out) return terr(SAXS_E_INVALID, "null argument");
  *out = nullptr;
  if (format == SAXS_TRAJ_AUTO) {
    const std::string s(path);
    auto ends = [&](const char *e) {
      const size_t n = std::strlen(e);
      if (s.size() < n) return false;
      for (size_t i = 0; i < n; ++i)
        if (std::tolower(static_cast<unsigned char>(s[s.size() - n + i])) != e[i]) return false;
      return true;
    };
    format = ends(".trr") ? SAXS_TRAJ_TRR : ends(".dcd") ? SAXS_TRAJ_DCD : ends(".xtc") ? SAXS_TRAJ_XTC : 0;
    if (!format) return terr(SAXS_E_INVALID, std::string("unsupported trajectory format: ") + path);
  }
  if (format != SAXS_TRAJ_TRR && format != SAXS_TRAJ_DCD && format != SAXS_TRAJ_XTC)
    return terr(SAXS_E_INVALID, "unknown trajectory format code");
  const int fd = ::open(path, O_RDONLY);
  if (fd < 0) return terr(SAXS_E_INVALID, std::string("cannot open ") + path);
  SaxsTraj *t = new SaxsTraj();
  t->fd = fd;
  t->format = format;
  const int rc = format == SAXS_TRAJ_TRR ? open_trr(t) : format == SAXS_TRAJ_DCD ? open_dcd(t) : open_xtc(t);
  if (rc) {
    ::close(fd);
    delete t;
    return rc;
  }
  *out = t;
  return SAXS_OK;
}

int saxs_traj_info(const SaxsTraj *t, int *natoms, long long *nframes) {
  if (!t) return terr(SAXS_E_INVALID, "null trajectory");
  if (natoms) *natoms = t->natoms;
  if (nframes) *nframes = static_cast<long long>(t->offsets.size());
  return SAXS_OK;
}

int saxs_traj_read(SaxsTraj *t, long long frame, float *xyz, float *box, double *time_ps) {
  if (!t || !xyz || !box) return terr(SAXS_E_INVALID, "null argument");
  if (frame < 0 || frame >= static_cast<long long>(t->offsets.size()))
    return terr(SAXS_E_RANGE, "frame " + std::to_string(frame) + " out of range [0, " +
                                  std::to_string(t->offsets.size()) + ")");
  if (t->format == SAXS_TRAJ_TRR) return read_trr(t, frame, xyz, box, time_ps);
  if (t->format == SAXS_TRAJ_DCD) return read_dcd(t, frame, xyz, box, time_ps);
  return read_xtc(t, frame, xyz, box, time_ps);
}

void saxs_traj_close(SaxsTraj *t) {
  if (!t) return;
  if (t->fd >= 0) ::close(t->fd);
  delete t;
}

}  // extern "C"
