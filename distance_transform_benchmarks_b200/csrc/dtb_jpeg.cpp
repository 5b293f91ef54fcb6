// dtb_jpeg.cpp -- JPEG files for dtb_image_read.  The reference's dt::imread (dt/src/imread.cpp:10-31) reads its
// benchmark inputs, gray JPEG photographs (benchmarks/distance_transform.cpp:55-74), through the JPEG decoder of
// stb_image (stbi_load; dt/src/stb_image.h, vendored by the reference) and rejects any file that is not
// 1-component.
//
// Format: ITU-T T.81 (ISO/IEC 10918-1) with the JFIF and Adobe colour conventions.  Read: Huffman-coded DCT,
// sequential (SOF0 baseline, SOF1 extended) and progressive (SOF2: spectral selection and successive
// approximation, T.81 Annex G) frames of 8-bit samples, 1 or 3 components with sampling factors 1-4 that divide
// the largest, restart intervals.  Arithmetic coding, 12-bit samples, lossless and hierarchical frames and
// 4-component (CMYK) files are rejected.
//
// Gray output is the reference's, byte for byte: coefficients are dequantised into 16-bit integers (truncated, as
// stb_image stores them: at decode time in sequential frames, after the last scan in progressive ones), and each
// 8x8 block goes through the Loeffler-Ligtenberg-Moschytz inverse DCT (the factorisation of the IJG "islow"
// transform) in integers at 12 fractional bits: columns first, keeping 2 extra bits ((x + 2^9) >> 10), then rows
// ((x + 2^16 + 128 * 2^17) >> 17, clamped to 0..255).  Integer products are exact, so the result depends only on
// the twelve rotation constants (formed as (int)(c * 4096 + 0.5), the rounding stb_image uses, which truncates the
// negative ones toward zero) and on those two rounding steps -- not on how the sums are grouped.  Where the
// reference's decoder would overflow 32-bit integers (only on corrupt coefficient data) this one computes in 64
// bits and may differ.
//
// Colour (3 components, read with channels = 3; the reference reads gray files only): chroma upsampled by the
// centred triangle filter for 2x factors (JFIF siting, as libjpeg's and stb_image's "fancy" upsampling) and by
// replication for other factors, then JFIF YCbCr -> RGB in 16-bit fixed point; files marked RGB (component ids
// 'R', 'G', 'B', or an Adobe marker with transform 0 and no JFIF marker) are copied.  Within a few levels of
// stb_image's RGB output; not claimed bit-exact.
#include <algorithm>
#include <cstring>
#include <vector>

#include "dtb_imgfile.h"

namespace dtb_io {
namespace {

constexpr int kFastBits = 9;        // Huffman codes up to this length decode with one table lookup
constexpr int kEndOfData = 0x100;   // "marker" met when the file ends inside entropy-coded data

// Natural (row-major) index of the k-th coefficient in zigzag order (T.81 Figure A.6), from the anti-diagonals.
struct Zigzag {
  uint8_t pos[64];
  Zigzag() {
    int k = 0;
    for (int s = 0; s < 15; ++s) {  // anti-diagonal x + y = s
      const int lo = s < 8 ? 0 : s - 7, hi = s < 8 ? s : 7;
      for (int i = 0; i <= hi - lo; ++i) {
        const int y = (s & 1) ? lo + i : hi - i;  // odd diagonals run down-left, even ones up-right
        pos[k++] = (uint8_t)(y * 8 + (s - y));
      }
    }
  }
};
const Zigzag kZz;

// Canonical Huffman table (T.81 Annex C; decoding per Annex F.2.2.3 with a lookup for the short codes).
struct Huffman {
  bool defined = false;
  uint16_t fast[1 << kFastBits];  // (length << 8) | symbol for codes of <= kFastBits bits, 0 for longer prefixes
  int32_t maxcode[17];            // largest code of each length 1-16, -1 when the length has none
  int32_t delta[17];              // index into vals of a code of that length, minus the code
  uint8_t vals[256];
  // AC coefficients whose code and magnitude bits both fit in the lookup: value, zero run and bits consumed
  // (0 = not in the lookup)
  int16_t ac_value[1 << kFastBits];
  uint8_t ac_run[1 << kFastBits];
  uint8_t ac_bits[1 << kFastBits];
};

bool build_huffman(Huffman& h, const uint8_t counts[16], const uint8_t* vals, int nvals) {
  std::memset(h.fast, 0, sizeof(h.fast));
  std::memcpy(h.vals, vals, (size_t)nvals);
  uint32_t code = 0;
  int k = 0;
  for (int len = 1; len <= 16; ++len) {
    const uint32_t n = counts[len - 1];
    if (code + n > (1u << len)) return false;  // more codes than this length holds
    h.delta[len] = k - (int32_t)code;
    h.maxcode[len] = n ? (int32_t)(code + n - 1) : -1;
    for (uint32_t i = 0; i < n; ++i, ++code, ++k)
      if (len <= kFastBits) {
        const uint32_t first = code << (kFastBits - len), cnt = 1u << (kFastBits - len);
        for (uint32_t j = 0; j < cnt; ++j) h.fast[first + j] = (uint16_t)(len << 8 | vals[k]);
      }
    code <<= 1;
  }
  for (uint32_t i = 0; i < (1u << kFastBits); ++i) {
    h.ac_bits[i] = 0;
    const uint16_t e = h.fast[i];
    const int len = e >> 8, s = e & 15, total = len + s;
    if (!e || !s || total > kFastBits) continue;
    const int v = (int)(i >> (kFastBits - total)) & ((1 << s) - 1);
    h.ac_value[i] = (int16_t)(v < (1 << (s - 1)) ? v - (1 << s) + 1 : v);  // T.81 F.2.2.1 EXTEND
    h.ac_run[i] = (uint8_t)((e & 0xFF) >> 4);
    h.ac_bits[i] = (uint8_t)total;
  }
  h.defined = true;
  return true;
}

// Entropy-coded data: byte stuffing (0xFF 0x00) removed, stops at the first marker and supplies zero bits past it.
struct BitReader {
  const uint8_t* p = nullptr;
  const uint8_t* end = nullptr;
  uint64_t buf = 0;  // the next bits, most significant first
  int nbits = 0;
  int marker = 0;    // marker code met (0 = none yet, kEndOfData at the file's end)

  void fill() {
    if (!marker && end - p >= 8) {  // eight bytes without 0xFF: no stuffing, no marker, append them at once
      uint64_t v;
      std::memcpy(&v, p, 8);
      const uint64_t x = ~v;  // 0xFF bytes become zero bytes
      if (!((x - 0x0101010101010101ull) & ~x & 0x8080808080808080ull)) {
        const int take = (64 - nbits) >> 3;
        v = __builtin_bswap64(v) >> nbits;
        if (nbits + 8 * take < 64) v &= ~0ull << (64 - nbits - 8 * take);
        buf |= v;
        nbits += 8 * take;
        p += take;
        return;
      }
    }
    while (nbits <= 56) {
      uint32_t byte = 0;
      if (!marker) {
        if (p >= end) {
          marker = kEndOfData;
        } else if ((byte = *p++) == 0xFF) {
          while (p < end && *p == 0xFF) ++p;  // fill bytes before a marker
          if (p < end && *p == 0x00) {
            ++p;                              // stuffed zero: 0xFF is data
          } else {
            marker = p < end ? *p++ : kEndOfData;
            byte = 0;
          }
        }
      }
      buf |= (uint64_t)byte << (56 - nbits);
      nbits += 8;
    }
  }
  void skip(int n) {
    buf <<= n;
    nbits -= n;
  }
  uint32_t bits(int n) {  // 0 <= n <= 16
    if (n == 0) return 0;
    if (nbits < n) fill();
    const uint32_t v = (uint32_t)(buf >> (64 - n));
    skip(n);
    return v;
  }
  // T.81 F.2.2.1 RECEIVE + EXTEND: an n-bit magnitude category value.
  int extend(int n) {
    const int v = (int)bits(n);
    return (n && v < (1 << (n - 1))) ? v - (1 << n) + 1 : v;
  }
  int decode(const Huffman& h) {  // the symbol, or -1 for a bit string that is no code of the table
    if (nbits < 16) fill();
    const uint16_t f = h.fast[buf >> (64 - kFastBits)];
    if (f) {
      skip(f >> 8);
      return f & 0xFF;
    }
    const uint32_t w = (uint32_t)(buf >> 48);
    for (int len = kFastBits + 1; len <= 16; ++len) {
      const int32_t code = (int32_t)(w >> (16 - len));
      if (code <= h.maxcode[len]) {
        skip(len);
        return h.vals[h.delta[len] + code];
      }
    }
    return -1;
  }
  // Moves to the next marker (past any data and fill bytes) unless one was met already.
  void find_marker() {
    while (!marker && p < end) {
      if (*p++ != 0xFF) continue;
      while (p < end && *p == 0xFF) ++p;
      if (p < end && *p != 0x00) marker = *p;
      if (p < end) ++p;
    }
    if (!marker) marker = kEndOfData;
  }
  // End of a restart interval: drops the buffered bits and steps over the RSTm marker.  False when the next
  // marker is not a restart marker (the scan's remaining data is missing).
  bool restart() {
    buf = 0;
    nbits = 0;
    find_marker();
    if (marker < 0xD0 || marker > 0xD7) return false;
    marker = 0;
    return true;
  }
};

struct Component {
  int id = 0, h = 1, v = 1, tq = 0;
  int td = 0, ta = 0;  // Huffman tables of the current scan
  int bw = 0, bh = 0;  // blocks stored: the MCU-padded grid
  int cw = 0, ch = 0;  // samples: ceil(X * h / hmax) x ceil(Y * v / vmax)
  int32_t dc_pred = 0;
  std::vector<int16_t> coef;    // progressive frames: bw * bh blocks of 64 raw coefficients, natural order
  std::vector<uint8_t> plane;   // samples, (bw * 8) x (bh * 8), row stride bw * 8
  int16_t* block(int bx, int by) { return &coef[((size_t)by * (size_t)bw + (size_t)bx) * 64]; }
  uint8_t* samples_at(int bx, int by) { return &plane[((size_t)by * (size_t)bw * 8 + (size_t)bx) * 8]; }
};

// The 8-point inverse DCT of the LLM factorisation on values scaled by 2^12 (c_k = cos(k pi / 16)):
// even part a rotation of (s2, s6) by sqrt2 c6 / sqrt2 (c2 - c6) / -sqrt2 (c2 + c6) and a butterfly of (s0, s4);
// odd part the four-input rotation network.  out[i] = (even +- odd + bias) >> shift, i and 7 - i.
constexpr int fix12(double c) { return (int)(c * 4096 + 0.5); }
constexpr int64_t K0541 = fix12(0.5411961), KM1847 = fix12(-1.847759065), K0765 = fix12(0.765366865);
constexpr int64_t K1175 = fix12(1.175875602), K0298 = fix12(0.298631336), K2053 = fix12(2.053119869);
constexpr int64_t K3072 = fix12(3.072711026), K1501 = fix12(1.501321110), KM0899 = fix12(-0.899976223);
constexpr int64_t KM2562 = fix12(-2.562915447), KM1961 = fix12(-1.961570560), KM0390 = fix12(-0.390180644);
static_assert(KM1847 == -7567 && KM0899 == -3685 && K0541 == 2217, "constants formed as the reference's decoder");

inline void idct8(const int64_t s[8], int64_t bias, int shift, int64_t out[8]) {
  const int64_t z1 = (s[2] + s[6]) * K0541;
  const int64_t e2 = z1 + s[6] * KM1847, e3 = z1 + s[2] * K0765;
  const int64_t e0 = (s[0] + s[4]) * 4096 + bias, e1 = (s[0] - s[4]) * 4096 + bias;
  const int64_t a0 = e0 + e3, a3 = e0 - e3, a1 = e1 + e2, a2 = e1 - e2;
  const int64_t z13 = s[7] + s[3], z24 = s[5] + s[1], z14 = s[7] + s[1], z23 = s[5] + s[3];
  const int64_t z5 = (z13 + z24) * K1175;
  const int64_t r14 = z5 + z14 * KM0899, r23 = z5 + z23 * KM2562, r13 = z13 * KM1961, r24 = z24 * KM0390;
  const int64_t b0 = s[7] * K0298 + r14 + r13, b1 = s[5] * K2053 + r23 + r24;
  const int64_t b2 = s[3] * K3072 + r23 + r13, b3 = s[1] * K1501 + r14 + r24;
  out[0] = (a0 + b3) >> shift;
  out[7] = (a0 - b3) >> shift;
  out[1] = (a1 + b2) >> shift;
  out[6] = (a1 - b2) >> shift;
  out[2] = (a2 + b1) >> shift;
  out[5] = (a2 - b1) >> shift;
  out[3] = (a3 + b0) >> shift;
  out[4] = (a3 - b0) >> shift;
}

// One dequantised block to 8x8 samples at `dst` (row stride `stride`).
void idct_block(const int16_t* c, uint8_t* dst, size_t stride) {
  int64_t mid[64], s[8], o[8];
  for (int x = 0; x < 8; ++x) {  // columns, 2 extra bits kept
    for (int i = 0; i < 8; ++i) s[i] = c[i * 8 + x];
    idct8(s, 512, 10, o);
    for (int i = 0; i < 8; ++i) mid[i * 8 + x] = o[i];
  }
  for (int y = 0; y < 8; ++y) {  // rows: remove 2^17, round, level shift by 128
    idct8(&mid[y * 8], 65536 + (128 << 17), 17, o);
    for (int i = 0; i < 8; ++i) dst[(size_t)y * stride + i] = (uint8_t)std::clamp<int64_t>(o[i], 0, 255);
  }
}

inline int16_t dequant(int32_t coef, uint16_t q) { return (int16_t)(uint16_t)((uint32_t)coef * q); }

struct Decoder {
  const uint8_t* f;
  size_t size;
  size_t pos = 0;
  uint16_t q[4][64] = {};  // quantisation tables, natural order
  Huffman dc[4], ac[4];
  Component comp[3];
  int ncomp = 0, X = 0, Y = 0, hmax = 1, vmax = 1, mcux = 0, mcuy = 0;
  bool frame = false, progressive = false, jfif = false;
  int adobe_transform = -1, restart_interval = 0, eobrun = 0;

  Decoder(const uint8_t* file, size_t n) : f(file), size(n) {}

  int u8(size_t at) const { return f[at]; }
  int u16(size_t at) const { return f[at] << 8 | f[at + 1]; }

  // Body [at, at + len) of the marker segment that starts at pos; advances pos past it.
  bool segment(size_t& at, size_t& len) {
    if (pos + 2 > size) return false;
    const size_t L = (size_t)u16(pos);
    if (L < 2 || pos + L > size) return false;
    at = pos + 2;
    len = L - 2;
    pos += L;
    return true;
  }

  bool read_dqt(size_t at, size_t len) {
    while (len > 0) {
      const int pq = u8(at) >> 4, tq = u8(at) & 15;
      const size_t need = 1 + 64 * (size_t)(pq + 1);
      if (pq > 1 || tq > 3 || len < need) return false;
      for (int k = 0; k < 64; ++k) q[tq][kZz.pos[k]] = (uint16_t)(pq ? u16(at + 1 + 2 * k) : u8(at + 1 + k));
      at += need;
      len -= need;
    }
    return true;
  }

  bool read_dht(size_t at, size_t len) {
    while (len > 0) {
      if (len < 17) return false;
      const int tc = u8(at) >> 4, th = u8(at) & 15;
      uint8_t counts[16];
      int n = 0;
      for (int i = 0; i < 16; ++i) n += counts[i] = f[at + 1 + i];
      if (tc > 1 || th > 3 || n > 256 || len < 17 + (size_t)n) return false;
      if (!build_huffman(tc ? ac[th] : dc[th], counts, f + at + 17, n)) return false;
      at += 17 + n;
      len -= 17 + n;
    }
    return true;
  }

  bool read_sof(size_t at, size_t len) {
    if (frame || len < 6) return false;
    frame = true;
    Y = u16(at + 1);
    X = u16(at + 3);
    ncomp = u8(at + 5);
    if (u8(at) != 8 || X == 0 || Y == 0 || (ncomp != 1 && ncomp != 3) || len < 6 + 3 * (size_t)ncomp) return false;
    if ((uint64_t)X * (uint64_t)Y > kMaxFilePixels) return false;
    for (int i = 0; i < ncomp; ++i) {
      Component& c = comp[i];
      c.id = u8(at + 6 + 3 * i);
      c.h = u8(at + 7 + 3 * i) >> 4;
      c.v = u8(at + 7 + 3 * i) & 15;
      c.tq = u8(at + 8 + 3 * i);
      if (c.h < 1 || c.h > 4 || c.v < 1 || c.v > 4 || c.tq > 3) return false;
      hmax = std::max(hmax, c.h);
      vmax = std::max(vmax, c.v);
    }
    mcux = (X + 8 * hmax - 1) / (8 * hmax);
    mcuy = (Y + 8 * vmax - 1) / (8 * vmax);
    for (int i = 0; i < ncomp; ++i) {
      Component& c = comp[i];
      if (hmax % c.h || vmax % c.v) return false;  // non-integer chroma factors
      c.bw = mcux * c.h;
      c.bh = mcuy * c.v;
      c.cw = (int)(((int64_t)X * c.h + hmax - 1) / hmax);
      c.ch = (int)(((int64_t)Y * c.v + vmax - 1) / vmax);
      c.plane.assign((size_t)c.bw * (size_t)c.bh * 64, 0);
      if (progressive) c.coef.assign((size_t)c.bw * (size_t)c.bh * 64, 0);
    }
    return true;
  }

  // Sequential block (T.81 F.2.2): DC difference, then run / size pairs to the end of block; dequantised as decoded.
  bool block_sequential(BitReader& br, Component& c, int16_t* blk) {
    std::memset(blk, 0, 64 * sizeof(int16_t));
    const uint16_t* qt = q[c.tq];
    const Huffman& ht = ac[c.ta];
    const int t = br.decode(dc[c.td]);
    if (t < 0 || t > 15) return false;
    c.dc_pred = (int32_t)((uint32_t)c.dc_pred + (uint32_t)(t ? br.extend(t) : 0));
    blk[0] = dequant(c.dc_pred, qt[0]);
    for (int k = 1; k < 64;) {
      if (br.nbits < 16) br.fill();
      const uint32_t look = (uint32_t)(br.buf >> (64 - kFastBits));
      if (ht.ac_bits[look]) {  // code and magnitude in one lookup
        k += ht.ac_run[look];
        br.skip(ht.ac_bits[look]);
        const int at = k < 64 ? kZz.pos[k] : 63;
        blk[at] = dequant(ht.ac_value[look], qt[at]);
        ++k;
        continue;
      }
      const int rs = br.decode(ht);
      if (rs < 0) return false;
      const int r = rs >> 4, s = rs & 15;
      if (s == 0) {
        if (rs != 0xF0) break;  // end of block
        k += 16;                // sixteen zeros
        continue;
      }
      k += r;
      const int at = k < 64 ? kZz.pos[k] : 63;  // a corrupt run past the block's end lands on the last coefficient
      blk[at] = dequant(br.extend(s), qt[at]);
      ++k;
    }
    return true;
  }

  // Progressive DC scans (T.81 G.1.2.1): first scan codes the difference of the value >> Al; refinements add bit Al.
  bool block_dc(BitReader& br, Component& c, int16_t* blk, int ah, int al) {
    if (ah == 0) {
      const int t = br.decode(dc[c.td]);
      if (t < 0 || t > 15) return false;
      c.dc_pred = (int32_t)((uint32_t)c.dc_pred + (uint32_t)(t ? br.extend(t) : 0));
      blk[0] = (int16_t)(uint16_t)((uint32_t)c.dc_pred << al);
    } else if (br.bits(1)) {
      blk[0] = (int16_t)(blk[0] | (1 << al));
    }
    return true;
  }

  // Progressive AC first scan (T.81 G.1.2.2): band ss..se of one component, end-of-band runs across blocks.
  bool block_ac_first(BitReader& br, Component& c, int16_t* blk, int ss, int se, int al) {
    if (eobrun > 0) {
      --eobrun;
      return true;
    }
    const Huffman& ht = ac[c.ta];
    for (int k = ss; k <= se;) {
      if (br.nbits < 16) br.fill();
      const uint32_t look = (uint32_t)(br.buf >> (64 - kFastBits));
      if (ht.ac_bits[look]) {
        k += ht.ac_run[look];
        br.skip(ht.ac_bits[look]);
        blk[k < 64 ? kZz.pos[k] : 63] = (int16_t)(uint16_t)((uint32_t)(int32_t)ht.ac_value[look] << al);
        ++k;
        continue;
      }
      const int rs = br.decode(ht);
      if (rs < 0) return false;
      const int r = rs >> 4, s = rs & 15;
      if (s == 0) {
        if (r < 15) {  // end-of-band run of 2^r + (r more bits) blocks, this one included
          eobrun = (1 << r) - 1 + (int)br.bits(r);
          break;
        }
        k += 16;
        continue;
      }
      k += r;
      blk[k < 64 ? kZz.pos[k] : 63] = (int16_t)(uint16_t)((uint32_t)br.extend(s) << al);
      ++k;
    }
    return true;
  }

  // Progressive AC refinement (T.81 G.1.2.3): one correction bit for every coefficient already non-zero, new
  // coefficients of magnitude 2^Al placed after `r` zero-history coefficients.
  bool block_ac_refine(BitReader& br, Component& c, int16_t* blk, int ss, int se, int al) {
    const int p1 = 1 << al, m1 = -p1;
    auto correct = [&](int16_t& v) {
      if (br.bits(1) && (v & p1) == 0) v = (int16_t)(v + (v >= 0 ? p1 : m1));
    };
    int k = ss;
    if (eobrun == 0) {
      for (; k <= se; ++k) {
        const int rs = br.decode(ac[c.ta]);
        if (rs < 0) return false;
        int r = rs >> 4;
        const int s = rs & 15;
        int val = 0;
        if (s) {
          if (s != 1) return false;  // refinement values have magnitude 1
          val = br.bits(1) ? p1 : m1;
        } else if (r != 15) {        // end-of-band run, this block's remaining coefficients included
          eobrun = (1 << r) + (int)br.bits(r);
          break;
        }
        // step over r zero-history coefficients (correcting the non-zero ones met on the way)
        for (; k <= se; ++k) {
          int16_t& v = blk[kZz.pos[k]];
          if (v != 0) {
            correct(v);
          } else if (r-- == 0) {
            break;
          }
        }
        if (val && k <= se) blk[kZz.pos[k]] = (int16_t)val;
      }
    }
    if (eobrun > 0) {
      for (; k <= se; ++k) {
        int16_t& v = blk[kZz.pos[k]];
        if (v != 0) correct(v);
      }
      --eobrun;
    }
    return true;
  }

  bool read_scan(size_t at, size_t len) {
    if (!frame || len < 1) return false;
    const int ns = u8(at);
    if (ns < 1 || ns > ncomp || len != 4 + 2 * (size_t)ns) return false;
    int sc[3];
    int units = 0;
    for (int i = 0; i < ns; ++i) {
      const int id = u8(at + 1 + 2 * i), tt = u8(at + 2 + 2 * i);
      int j = 0;
      while (j < ncomp && comp[j].id != id) ++j;
      if (j == ncomp || (tt >> 4) > 3 || (tt & 15) > 3) return false;
      for (int m = 0; m < i; ++m)
        if (sc[m] == j) return false;
      sc[i] = j;
      comp[j].td = tt >> 4;
      comp[j].ta = tt & 15;
      units += comp[j].h * comp[j].v;
    }
    const int ss = u8(at + 1 + 2 * ns), se = u8(at + 2 + 2 * ns);
    const int ah = u8(at + 3 + 2 * ns) >> 4, al = u8(at + 3 + 2 * ns) & 15;
    if (ns > 1 && units > 10) return false;  // T.81 B.2.3: at most 10 blocks per MCU
    if (progressive) {
      if (ss > se || se > 63 || (ss == 0 && se != 0) || (ss > 0 && ns != 1) || ah > 13 || al > 13) return false;
    }
    for (int i = 0; i < ns; ++i) {
      const Component& c = comp[sc[i]];
      const bool need_dc = !progressive || (ss == 0 && ah == 0), need_ac = !progressive || ss > 0;
      if ((need_dc && !dc[c.td].defined) || (need_ac && !ac[c.ta].defined)) return false;
    }

    BitReader br;
    br.p = f + pos;
    br.end = f + size;
    for (int i = 0; i < ns; ++i) comp[sc[i]].dc_pred = 0;
    eobrun = 0;
    int16_t seq[64];
    auto unit = [&](Component& c, int bx, int by) {
      if (!progressive) {  // sequential: samples straight away, while the block is in cache
        if (!block_sequential(br, c, seq)) return false;
        idct_block(seq, c.samples_at(bx, by), (size_t)c.bw * 8);
        return true;
      }
      int16_t* blk = c.block(bx, by);
      if (ss == 0) return block_dc(br, c, blk, ah, al);
      return ah == 0 ? block_ac_first(br, c, blk, ss, se, al) : block_ac_refine(br, c, blk, ss, se, al);
    };
    // A one-component scan codes its component's own blocks one by one (T.81 A.2.2); an interleaved scan codes
    // MCUs of h x v blocks per component.
    const int ux = ns == 1 ? (comp[sc[0]].cw + 7) / 8 : mcux, uy = ns == 1 ? (comp[sc[0]].ch + 7) / 8 : mcuy;
    int todo = restart_interval;
    bool done = false;
    for (int my = 0; my < uy && !done; ++my)
      for (int mx = 0; mx < ux && !done; ++mx) {
        if (ns == 1) {
          if (!unit(comp[sc[0]], mx, my)) return false;
        } else {
          for (int i = 0; i < ns; ++i) {
            Component& c = comp[sc[i]];
            for (int v = 0; v < c.v; ++v)
              for (int h = 0; h < c.h; ++h)
                if (!unit(c, mx * c.h + h, my * c.v + v)) return false;
          }
        }
        if (restart_interval && --todo == 0 && !(my == uy - 1 && mx == ux - 1)) {
          todo = restart_interval;
          if (!br.restart()) {
            done = true;  // no RSTm where one belongs: the rest of the scan stays zero
          } else {
            for (int i = 0; i < ns; ++i) comp[sc[i]].dc_pred = 0;
            eobrun = 0;
          }
        }
      }
    br.find_marker();  // the byte after the scan's data: a marker code
    pos = br.marker == kEndOfData ? size : (size_t)(br.p - f) - 2;
    return true;
  }

  bool parse() {
    if (size < 4 || f[0] != 0xFF || f[1] != 0xD8) return false;
    pos = 2;
    bool scanned = false;
    while (pos < size) {
      if (f[pos] != 0xFF) {  // junk between segments: look for the next marker
        ++pos;
        continue;
      }
      while (pos < size && f[pos] == 0xFF) ++pos;  // fill bytes
      if (pos >= size) break;
      const int m = f[pos++];
      if (m == 0xD9) break;                            // EOI
      if (m == 0x00 || m == 0x01 || (m >= 0xD0 && m <= 0xD8)) continue;  // no segment follows
      size_t at, len;
      if (!segment(at, len)) return scanned;
      switch (m) {
        case 0xC0:
        case 0xC1:
        case 0xC2:
          progressive = m == 0xC2;
          if (!read_sof(at, len)) return false;
          break;
        case 0xC4:
          if (!read_dht(at, len)) return false;
          break;
        case 0xDB:
          if (!read_dqt(at, len)) return false;
          break;
        case 0xDD:
          if (len < 2) return false;
          restart_interval = u16(at);
          break;
        case 0xDA:
          if (!read_scan(at, len)) return false;
          scanned = true;
          break;
        case 0xE0:
          if (len >= 5 && std::memcmp(f + at, "JFIF\0", 5) == 0) jfif = true;
          break;
        case 0xEE:
          if (len >= 12 && std::memcmp(f + at, "Adobe", 5) == 0) adobe_transform = u8(at + 11);
          break;
        default:
          if ((m >= 0xC3 && m <= 0xCF && m != 0xC4 && m != 0xC8 && m != 0xCC))
            return false;  // lossless, hierarchical, arithmetic-coded or 12-bit frames
          break;             // APPn, COM, DNL and the rest: skipped
      }
    }
    return frame && scanned;
  }

  // Progressive frames: dequantise the coefficients (the tables in force after the last scan) and transform the
  // blocks that hold samples of the component.
  void finish_progressive(Component& c) {
    const int nx = (c.cw + 7) / 8, ny = (c.ch + 7) / 8;
    for (int by = 0; by < ny; ++by)
      for (int bx = 0; bx < nx; ++bx) {
        int16_t* blk = c.block(bx, by);
        for (int i = 0; i < 64; ++i) blk[i] = dequant(blk[i], q[c.tq][i]);
        idct_block(blk, c.samples_at(bx, by), (size_t)c.bw * 8);
      }
  }

  // Component c at full resolution, X x Y: triangle filter for 2x factors, replication otherwise.
  std::vector<uint8_t> upsample(const Component& c) {
    const std::vector<uint8_t>& plane = c.plane;
    const size_t stride = (size_t)c.bw * 8;
    const int hs = hmax / c.h, vs = vmax / c.v;
    std::vector<uint8_t> out((size_t)X * Y);
    if (hs > 2 || vs > 2) {
      for (int y = 0; y < Y; ++y)
        for (int x = 0; x < X; ++x) out[(size_t)y * X + x] = plane[(size_t)(y / vs) * stride + (size_t)(x / hs)];
      return out;
    }
    std::vector<int> t((size_t)c.cw);
    for (int y = 0; y < Y; ++y) {
      // vertical: 4 * sample, or 3 * nearer + farther source row (JFIF siting between the two)
      const int near = y / vs;
      const int far = vs == 1 ? near : std::clamp(near + ((y & 1) ? 1 : -1), 0, c.ch - 1);
      const uint8_t* rn = &plane[(size_t)near * stride];
      const uint8_t* rf = &plane[(size_t)far * stride];
      for (int i = 0; i < c.cw; ++i) t[i] = vs == 1 ? 4 * rn[i] : 3 * rn[i] + rf[i];
      uint8_t* o = &out[(size_t)y * X];
      if (hs == 1) {
        for (int x = 0; x < X; ++x) o[x] = (uint8_t)((t[x] + 2) >> 2);
      } else {
        for (int x = 0; x < X; ++x) {
          const int i = x >> 1, j = std::clamp(i + ((x & 1) ? 1 : -1), 0, c.cw - 1);
          o[x] = (uint8_t)((3 * t[i] + t[j] + 8) >> 4);
        }
        // stb_image's horizontal-only filter weights the last even output 3:1 toward the second-to-last sample
        // (3 * in[w-2] + in[w-1]); kept so that 4:2:2 files match it on the right edge too
        if (vs == 1 && c.cw >= 2 && 2 * (c.cw - 1) < X)
          o[2 * (c.cw - 1)] = (uint8_t)((3 * t[c.cw - 2] + t[c.cw - 1] + 8) >> 4);
      }
    }
    return out;
  }

  void output(Pixels& out) {
    out.w = X;
    out.h = Y;
    out.channels = ncomp;
    if (progressive)
      for (int i = 0; i < ncomp; ++i) finish_progressive(comp[i]);
    if (ncomp == 1) {
      const std::vector<uint8_t>& plane = comp[0].plane;
      const size_t stride = (size_t)comp[0].bw * 8;
      out.data.resize((size_t)X * Y);
      for (int y = 0; y < Y; ++y) std::memcpy(&out.data[(size_t)y * X], &plane[(size_t)y * stride], (size_t)X);
      return;
    }
    std::vector<uint8_t> full[3];
    for (int i = 0; i < 3; ++i) full[i] = upsample(comp[i]);
    const bool rgb = (comp[0].id == 'R' && comp[1].id == 'G' && comp[2].id == 'B') ||
                     (adobe_transform == 0 && !jfif);
    out.data.resize((size_t)X * Y * 3);
    for (size_t i = 0; i < (size_t)X * Y; ++i) {
      uint8_t* o = &out.data[3 * i];
      if (rgb) {
        o[0] = full[0][i];
        o[1] = full[1][i];
        o[2] = full[2][i];
        continue;
      }
      // JFIF: R = Y + 1.402 Cr, G = Y - 0.344136 Cb - 0.714136 Cr, B = Y + 1.772 Cb (Cb, Cr centred on 128)
      const int yy = (full[0][i] << 16) + 32768, cb = full[1][i] - 128, cr = full[2][i] - 128;
      o[0] = (uint8_t)std::clamp((yy + 91881 * cr) >> 16, 0, 255);
      o[1] = (uint8_t)std::clamp((yy - 22554 * cb - 46802 * cr) >> 16, 0, 255);
      o[2] = (uint8_t)std::clamp((yy + 116130 * cb) >> 16, 0, 255);
    }
  }
};

}  // namespace

dtb_status decode_jpeg(const uint8_t* file, size_t size, Pixels& out) {
  Decoder d(file, size);
  if (!d.parse()) return DTB_ERR_INVALID_ARG;
  d.output(out);
  return DTB_OK;
}

}  // namespace dtb_io
