// meshoptimizer's vertex and index buffer codecs, as the reference's `.vgeo` writer uses them
// (src/core/io/serialize.ts:244 `encodeVertexBufferLevel(raw, count, stride, 2, 1)`, :290 `encodeIndexBuffer(slots,
// count, 4)`; read back at :338-346 and :369-388). meshoptimizer is an npm dependency of the reference that is not
// vendored with it; this file restates the two published stream formats (meshoptimizer's documented vertex codec,
// versions 0 and 1, and index codec, versions 0 and 1) in its own code. The decoders follow the formats; the
// encoders are this file's own (any encoder whose output the format decodes is valid: the reference itself decodes
// every candidate once and keeps it only when the bytes round-trip).
//
// Vertex stream: header 0xa0 | version; blocks of up to min(8192 / stride rounded down to 16, 256) vertices; a
// version-1 block starts with stride / 4 control bytes (2 bits per byte column: 0 / 1 = byte groups whose 2-bit
// headers pick {0, 1, 2, 4} / {1, 2, 4, 8} bits per value, 2 = all zero, 3 = the bytes as they are); version 0 has no
// control bytes and picks {0, 2, 4, 8}. Each byte column is the column's deltas: per byte (channel 0), per 16-bit
// word (channel 1) or a rotated xor of 32-bit words (channel 2), zigzag-coded, against the previous vertex (the
// first vertex of the buffer before the first block). A byte group holds 16 values: `bits` bits each, most
// significant first (1-bit groups least significant first), a value of all ones escaping to a full byte appended
// after the group. The stream ends with the first vertex and (version 1) the per-4-byte channel modes, padded in
// front with zeros to at least 32 (version 0) / 24 (version 1) bytes.
//
// Index stream: header 0xe0 | version; one code byte per triangle, then the data bytes, then a 16-byte table of
// "aux" codes. Decoding keeps a 16-entry FIFO of edges and one of vertices and the next new vertex: a code < 0xf0
// takes edge (code >> 4) of the FIFO and names the third vertex (code & 15: 0 = next new vertex, a vertex FIFO entry,
// or - version 1 - 13 / 14 = last free index -1 / +1, 15 = a free index in the data); codes 0xf0-0xfd take the aux
// code of the table, 0xfe / 0xff one from the data (the first vertex then the next new one / a free index); an aux
// code holds the other two vertices (0 = next new, 1-13 vertex FIFO entry - 1, 15 = free index). Free indices are
// zigzag deltas from the last free index, 7 bits per byte. Triangles come out rotated so that the matched edge or
// the new vertex leads.
#include <cstdint>
#include <cstring>
#include <vector>

#include "vgbuild.h"

namespace {

constexpr size_t kBlockBytes = 8192, kBlockMax = 256, kGroup = 16, kGroupDecodeLimit = 24;
constexpr size_t kTailMinV0 = 32, kTailMinV1 = 24;
constexpr int kBitsV0[4] = {0, 2, 4, 8};
constexpr int kBitsV1[5] = {0, 1, 2, 4, 8};

size_t block_vertices(size_t stride) {
  const size_t n = (kBlockBytes / stride) & ~(kGroup - 1);
  return n < kBlockMax ? n : kBlockMax;
}

uint32_t rotl(uint32_t v, int r) { return (v << r) | (v >> ((32 - r) & 31)); }

// ---- byte groups
const uint8_t *read_group(const uint8_t *data, uint8_t *out, int bits) {
  if (bits == 0) {
    std::memset(out, 0, kGroup);
    return data;
  }
  if (bits == 8) {
    std::memcpy(out, data, kGroup);
    return data + kGroup;
  }
  const int per_byte = 8 / bits;
  const uint8_t sentinel = uint8_t((1 << bits) - 1);
  const uint8_t *extra = data + kGroup / per_byte;
  for (size_t i = 0; i < kGroup; i++) {
    const uint8_t byte = data[i / per_byte];
    const int k = int(i % per_byte);
    const int shift = bits == 1 ? k : 8 - bits * (k + 1);
    uint8_t v = uint8_t((byte >> shift) & sentinel);
    if (v == sentinel) v = *extra++;
    out[i] = v;
  }
  return extra;
}

size_t group_size(const uint8_t *v, int bits) {
  if (bits == 0) {
    for (size_t i = 0; i < kGroup; i++)
      if (v[i]) return SIZE_MAX;
    return 0;
  }
  if (bits == 8) return kGroup;
  const uint8_t sentinel = uint8_t((1 << bits) - 1);
  size_t n = kGroup * bits / 8;
  for (size_t i = 0; i < kGroup; i++) n += v[i] >= sentinel;
  return n;
}

uint8_t *write_group(uint8_t *data, const uint8_t *v, int bits) {
  if (bits == 0) return data;
  if (bits == 8) {
    std::memcpy(data, v, kGroup);
    return data + kGroup;
  }
  const int per_byte = 8 / bits;
  const uint8_t sentinel = uint8_t((1 << bits) - 1);
  for (size_t b = 0; b < kGroup / per_byte; b++) {
    uint8_t byte = 0;
    for (int k = 0; k < per_byte; k++) {
      const uint8_t e = v[b * per_byte + k] >= sentinel ? sentinel : v[b * per_byte + k];
      const int shift = bits == 1 ? k : 8 - bits * (k + 1);
      byte = uint8_t(byte | (e << shift));
    }
    *data++ = byte;
  }
  for (size_t i = 0; i < kGroup; i++)
    if (v[i] >= sentinel) *data++ = v[i];
  return data;
}

// `n` (a multiple of 16) values as headed byte groups with the bit widths `bits`
const uint8_t *read_bytes(const uint8_t *data, const uint8_t *end, uint8_t *out, size_t n, const int *bits) {
  const size_t header = (n / kGroup + 3) / 4;
  if (size_t(end - data) < header) return nullptr;
  const uint8_t *head = data;
  data += header;
  for (size_t g = 0; g < n / kGroup; g++) {
    if (size_t(end - data) < kGroupDecodeLimit) return nullptr;
    const int k = (head[g / 4] >> ((g % 4) * 2)) & 3;
    data = read_group(data, out + g * kGroup, bits[k]);
  }
  return data;
}

size_t bytes_size(const uint8_t *v, size_t n, const int *bits, int *choice) {
  size_t total = (n / kGroup + 3) / 4;
  for (size_t g = 0; g < n / kGroup; g++) {
    size_t best = SIZE_MAX;
    int pick = 3;
    for (int k = 0; k < 4; k++) {
      const size_t s = group_size(v + g * kGroup, bits[k]);
      if (s < best) best = s, pick = k;
    }
    if (choice) choice[g] = pick;
    total += best;
  }
  return total;
}

uint8_t *write_bytes(uint8_t *data, const uint8_t *v, size_t n, const int *bits) {
  std::vector<int> choice(n / kGroup);
  bytes_size(v, n, bits, choice.data());
  const size_t header = (n / kGroup + 3) / 4;
  std::memset(data, 0, header);
  for (size_t g = 0; g < n / kGroup; g++) data[g / 4] = uint8_t(data[g / 4] | (choice[g] << ((g % 4) * 2)));
  data += header;
  for (size_t g = 0; g < n / kGroup; g++) data = write_group(data, v + g * kGroup, bits[choice[g]]);
  return data;
}

// ---- deltas of one 4-byte column group (bytes k0..k0+3 of every vertex of a block)
template <typename T>
T zigzag(T v) {
  return T((v << 1) ^ T(0 - (v >> (sizeof(T) * 8 - 1))));
}
template <typename T>
T unzigzag(T v) {
  return T((v >> 1) ^ T(0 - (v & 1)));
}

// cols[j][i]: byte j of the group's delta of vertex i
void encode_deltas(const uint8_t *src, size_t count, size_t stride, size_t k0, const uint8_t *last, int channel,
                   uint8_t (*cols)[kBlockMax]) {
  uint32_t p = 0;
  std::memcpy(&p, last + k0, 4);
  for (size_t i = 0; i < count; i++) {
    uint32_t v = 0;
    std::memcpy(&v, src + i * stride + k0, 4);
    uint32_t d;
    if ((channel & 3) == 0) {
      d = 0;
      for (int j = 0; j < 4; j++) d |= uint32_t(zigzag<uint8_t>(uint8_t((v >> (8 * j)) - (p >> (8 * j))))) << (8 * j);
    } else if ((channel & 3) == 1) {
      d = zigzag<uint16_t>(uint16_t(v - p)) | uint32_t(zigzag<uint16_t>(uint16_t((v >> 16) - (p >> 16)))) << 16;
    } else {
      d = rotl(v ^ p, channel >> 4);
    }
    for (int j = 0; j < 4; j++) cols[j][i] = uint8_t(d >> (8 * j));
    p = v;
  }
}

bool decode_deltas(uint8_t (*cols)[kBlockMax], size_t count, size_t stride, size_t k0, uint8_t *last, int channel,
                   uint8_t *dst) {
  if ((channel & 3) == 3) return false;
  uint32_t p = 0;
  std::memcpy(&p, last + k0, 4);
  for (size_t i = 0; i < count; i++) {
    const uint32_t d = uint32_t(cols[0][i]) | uint32_t(cols[1][i]) << 8 | uint32_t(cols[2][i]) << 16 |
                       uint32_t(cols[3][i]) << 24;
    uint32_t v;
    if ((channel & 3) == 0) {
      v = 0;
      for (int j = 0; j < 4; j++) v |= uint32_t(uint8_t(unzigzag<uint8_t>(uint8_t(d >> (8 * j))) + (p >> (8 * j)))) << (8 * j);
    } else if ((channel & 3) == 1) {
      v = uint32_t(uint16_t(unzigzag<uint16_t>(uint16_t(d)) + p)) |
          uint32_t(uint16_t(unzigzag<uint16_t>(uint16_t(d >> 16)) + (p >> 16))) << 16;
    } else {
      v = rotl(d, (32 - (channel >> 4)) & 31) ^ p;
    }
    std::memcpy(dst + i * stride + k0, &v, 4);
    p = v;
  }
  std::memcpy(last + k0, dst + (count - 1) * stride + k0, 4);
  return true;
}

size_t column_size(const uint8_t *col, size_t count, int version, int *ctrl) {
  const size_t aligned = (count + kGroup - 1) & ~(kGroup - 1);
  if (version == 0) {
    *ctrl = 0;
    return bytes_size(col, aligned, kBitsV0, nullptr);
  }
  bool zero = true;
  for (size_t i = 0; i < count; i++) zero = zero && col[i] == 0;
  if (zero) {
    *ctrl = 2;
    return 0;
  }
  size_t best = count;
  *ctrl = 3;
  for (int c = 0; c < 2; c++) {
    const size_t s = bytes_size(col, aligned, kBitsV1 + c, nullptr);
    if (s < best) best = s, *ctrl = c;
  }
  return best;
}

}  // namespace

extern "C" {

size_t vgb_vertex_encode_bound(size_t count, size_t stride) {
  const size_t bs = stride ? block_vertices(stride) : 1;
  const size_t blocks = bs ? (count + bs - 1) / bs : 0;
  const size_t aligned = (bs + kGroup - 1) & ~(kGroup - 1);
  const size_t per_block = stride / 4 + stride * ((aligned / kGroup + 3) / 4 + aligned);
  const size_t tail = stride + stride / 4 > kTailMinV0 ? stride + stride / 4 : kTailMinV0;
  return 1 + blocks * per_block + tail;
}

size_t vgb_vertex_encode(uint8_t *dst, size_t capacity, const void *vertices, size_t count, size_t stride,
                         int version) {
  if (!dst || (!vertices && count) || stride == 0 || stride > 256 || stride % 4 || (version != 0 && version != 1) ||
      capacity < vgb_vertex_encode_bound(count, stride))
    return 0;
  const uint8_t *src = static_cast<const uint8_t *>(vertices);
  uint8_t *out = dst;
  *out++ = uint8_t(0xa0 | version);
  uint8_t first[256] = {}, last[256] = {};
  if (count) std::memcpy(first, src, stride);
  std::memcpy(last, first, stride);
  // channel mode per 4-byte column group (version 1): the smaller of byte and 16-bit deltas over the buffer
  uint8_t channels[64] = {};
  const size_t bs = block_vertices(stride);
  static thread_local uint8_t cols[4][kBlockMax];
  if (version == 1) {
    for (size_t k0 = 0; k0 < stride; k0 += 4) {
      size_t size[2] = {0, 0};
      for (int ch = 0; ch < 2; ch++) {
        uint8_t prev[256];
        std::memcpy(prev, first, stride);
        for (size_t at = 0; at < count; at += bs) {
          const size_t n = count - at < bs ? count - at : bs;
          encode_deltas(src + at * stride, n, stride, k0, prev, ch, cols);
          for (int j = 0; j < 4; j++) {
            int c;
            size[ch] += column_size(cols[j], n, version, &c);
          }
          std::memcpy(prev + k0, src + (at + n - 1) * stride + k0, 4);
        }
      }
      channels[k0 / 4] = size[1] < size[0] ? 1 : 0;
    }
  }
  for (size_t at = 0; at < count; at += bs) {
    const size_t n = count - at < bs ? count - at : bs;
    const size_t aligned = (n + kGroup - 1) & ~(kGroup - 1);
    uint8_t *control = out;
    if (version == 1) {
      std::memset(control, 0, stride / 4);
      out += stride / 4;
    }
    for (size_t k0 = 0; k0 < stride; k0 += 4) {
      encode_deltas(src + at * stride, n, stride, k0, last, channels[k0 / 4], cols);
      for (int j = 0; j < 4; j++) {
        std::memset(cols[j] + n, 0, aligned - n);
        int ctrl = 0;
        column_size(cols[j], n, version, &ctrl);
        if (version == 1) control[k0 / 4] = uint8_t(control[k0 / 4] | (ctrl << (j * 2)));
        if (ctrl == 3) {
          std::memcpy(out, cols[j], n);
          out += n;
        } else if (ctrl != 2) {
          out = write_bytes(out, cols[j], aligned, version == 0 ? kBitsV0 : kBitsV1 + ctrl);
        }
      }
    }
    std::memcpy(last, src + (at + n - 1) * stride, stride);
  }
  const size_t tail = stride + (version == 1 ? stride / 4 : 0);
  const size_t tail_min = version == 0 ? kTailMinV0 : kTailMinV1;
  if (tail < tail_min) {
    std::memset(out, 0, tail_min - tail);
    out += tail_min - tail;
  }
  std::memcpy(out, first, stride);
  out += stride;
  if (version == 1) {
    std::memcpy(out, channels, stride / 4);
    out += stride / 4;
  }
  return size_t(out - dst);
}

int vgb_vertex_decode(void *vertices, size_t count, size_t stride, const uint8_t *src, size_t size) {
  if (!vertices || !src || stride == 0 || stride > 256 || stride % 4) return -4;
  const uint8_t *data = src, *end = src + size;
  if (size < 1) return -2;
  const uint8_t header = *data++;
  if ((header & 0xf0) != 0xa0) return -1;
  const int version = header & 15;
  if (version > 1) return -1;
  const size_t tail = stride + (version == 1 ? stride / 4 : 0);
  const size_t tail_min = version == 0 ? kTailMinV0 : kTailMinV1;
  const size_t tail_pad = tail < tail_min ? tail_min : tail;
  if (size_t(end - data) < tail_pad) return -2;
  uint8_t last[256];
  std::memcpy(last, end - tail, stride);
  const uint8_t *channels = version == 1 ? end - tail + stride : nullptr;
  uint8_t *dst = static_cast<uint8_t *>(vertices);
  const size_t bs = block_vertices(stride);
  uint8_t cols[4][kBlockMax];  // a column's groups fill at most 256 bytes
  for (size_t at = 0; at < count; at += bs) {
    const size_t n = count - at < bs ? count - at : bs;
    const size_t aligned = (n + kGroup - 1) & ~(kGroup - 1);
    const uint8_t *control = data;
    if (version == 1) {
      if (size_t(end - data) < stride / 4) return -2;
      data += stride / 4;
    }
    for (size_t k0 = 0; k0 < stride; k0 += 4) {
      const uint8_t cb = version == 1 ? control[k0 / 4] : 0;
      for (int j = 0; j < 4; j++) {
        const int ctrl = (cb >> (j * 2)) & 3;
        if (ctrl == 3) {
          if (size_t(end - data) < n) return -2;
          std::memcpy(cols[j], data, n);
          data += n;
        } else if (ctrl == 2) {
          std::memset(cols[j], 0, n);
        } else {
          data = read_bytes(data, end, cols[j], aligned, version == 0 ? kBitsV0 : kBitsV1 + ctrl);
          if (!data) return -2;
        }
      }
      if (!decode_deltas(cols, n, stride, k0, last, version == 1 ? channels[k0 / 4] : 0, dst + at * stride)) return -1;
    }
  }
  if (size_t(end - data) != tail_pad) return -3;
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------- index codec
namespace {

constexpr uint8_t kAuxTable[16] = {0x00, 0x76, 0x87, 0x56, 0x67, 0x78, 0xa9, 0x86,
                                   0x65, 0x89, 0x68, 0x98, 0x01, 0x69, 0x00, 0x00};

struct Fifos {
  uint32_t edge[16][2];
  uint32_t vert[16];
  uint32_t eo = 0, vo = 0;
  Fifos() {
    std::memset(edge, 0xff, sizeof edge);
    std::memset(vert, 0xff, sizeof vert);
  }
  void push_edge(uint32_t a, uint32_t b) {
    edge[eo][0] = a;
    edge[eo][1] = b;
    eo = (eo + 1) & 15;
  }
  void push_vert(uint32_t v, bool cond = true) {
    vert[vo] = v;
    vo = (vo + (cond ? 1 : 0)) & 15;
  }
  int find_vert(uint32_t v) const {
    for (int i = 0; i < 16; i++)
      if (vert[(vo - 1 - i) & 15] == v) return i;
    return -1;
  }
  // (fifo position << 2) | rotation of the triangle whose leading edge is in the FIFO, or -1
  int find_edge(uint32_t a, uint32_t b, uint32_t c) const {
    for (int i = 0; i < 16; i++) {
      const uint32_t *e = edge[(eo - 1 - i) & 15];
      if (e[0] == a && e[1] == b) return i << 2;
      if (e[0] == b && e[1] == c) return (i << 2) | 1;
      if (e[0] == c && e[1] == a) return (i << 2) | 2;
    }
    return -1;
  }
};

void put_index(uint8_t *&data, uint32_t index, uint32_t last) {
  const uint32_t d = index - last;
  uint32_t v = (d << 1) ^ uint32_t(int32_t(d) >> 31);
  do {
    *data++ = uint8_t((v & 127) | (v > 127 ? 128 : 0));
    v >>= 7;
  } while (v);
}

bool get_index(const uint8_t *&data, const uint8_t *end, uint32_t last, uint32_t &out) {
  uint32_t v = 0;
  for (int shift = 0; shift < 35; shift += 7) {
    if (data >= end) return false;
    const uint8_t g = *data++;
    v |= uint32_t(g & 127) << shift;
    if (g < 128) {
      out = last + ((v >> 1) ^ uint32_t(0 - (v & 1)));
      return true;
    }
  }
  return false;
}

constexpr int kOrder[3][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}};

}  // namespace

extern "C" {

size_t vgb_index_encode_bound(size_t index_count, size_t vertex_count) {
  int bits = 0;
  while (bits < 32 && (vertex_count >> bits)) bits++;
  const size_t vbytes = size_t((bits + 6) / 7);
  return 1 + index_count / 3 * (1 + 1 + 3 * (vbytes > 5 ? vbytes : 5)) + 16;
}

size_t vgb_index_encode(uint8_t *dst, size_t capacity, const uint32_t *indices, size_t index_count, int version) {
  if (!dst || (!indices && index_count) || index_count % 3 || (version != 0 && version != 1)) return 0;
  uint32_t vmax = 0;
  for (size_t i = 0; i < index_count; i++) vmax = indices[i] > vmax ? indices[i] : vmax;
  if (capacity < vgb_index_encode_bound(index_count, size_t(vmax) + 1)) return 0;
  Fifos f;
  uint32_t next = 0, last = 0;
  const int fecmax = version >= 1 ? 13 : 15;
  uint8_t *code = dst + 1;
  uint8_t *data = code + index_count / 3;
  dst[0] = uint8_t(0xe0 | version);
  for (size_t i = 0; i < index_count; i += 3) {
    const int fer = f.find_edge(indices[i], indices[i + 1], indices[i + 2]);
    if (fer >= 0 && (fer >> 2) < 15) {
      const int *o = kOrder[fer & 3];
      const uint32_t a = indices[i + o[0]], b = indices[i + o[1]], c = indices[i + o[2]];
      const int fe = fer >> 2;
      const int fc = f.find_vert(c);
      int fec = (fc >= 1 && fc < fecmax) ? fc : (c == next) ? (next++, 0) : 15;
      if (fec == 15 && version >= 1) {
        if (c + 1 == last) fec = 13, last = c;
        else if (c == last + 1) fec = 14, last = c;
      }
      *code++ = uint8_t((fe << 4) | fec);
      if (fec == 15) put_index(data, c, last), last = c;
      if (fec == 0 || fec >= fecmax) f.push_vert(c);
      f.push_edge(c, b);
      f.push_edge(a, c);
    } else {
      const int rot = indices[i + 1] == next ? 1 : indices[i + 2] == next ? 2 : 0;
      const int *o = kOrder[rot];
      const uint32_t a = indices[i + o[0]], b = indices[i + o[1]], c = indices[i + o[2]];
      bool reset = false;
      if (a == 0 && b == 1 && c == 2 && next > 0 && version >= 1) {
        reset = true;
        next = 0;
        std::memset(f.vert, 0xff, sizeof f.vert);  // old vertices are never named again
      }
      const int fb = f.find_vert(b), fc = f.find_vert(c);
      const int fea = (a == next) ? (next++, 0) : 15;
      const int feb = (fb >= 0 && fb < 14) ? fb + 1 : (b == next) ? (next++, 0) : 15;
      const int fec = (fc >= 0 && fc < 14) ? fc + 1 : (c == next) ? (next++, 0) : 15;
      const uint8_t aux = uint8_t((feb << 4) | fec);
      int ai = -1;
      for (int k = 0; k < 14 && ai < 0; k++)
        if (kAuxTable[k] == aux) ai = k;
      if (fea == 0 && ai >= 0 && !reset) {
        *code++ = uint8_t(0xf0 | ai);
      } else {
        *code++ = uint8_t(0xf0 | 14 | (fea == 15 ? 1 : 0));
        *data++ = aux;
      }
      if (fea == 15) put_index(data, a, last), last = a;
      if (feb == 15) put_index(data, b, last), last = b;
      if (fec == 15) put_index(data, c, last), last = c;
      f.push_vert(a);
      if (feb == 0 || feb == 15) f.push_vert(b);
      if (fec == 0 || fec == 15) f.push_vert(c);
      f.push_edge(b, a);
      f.push_edge(c, b);
      f.push_edge(a, c);
    }
  }
  std::memcpy(data, kAuxTable, 16);
  data += 16;
  return size_t(data - dst);
}

int vgb_index_decode(uint32_t *out, size_t index_count, const uint8_t *src, size_t size) {
  if (!out || !src || index_count % 3) return -4;
  if (size < 1 + index_count / 3 + 16) return -2;
  if ((src[0] & 0xf0) != 0xe0) return -1;
  const int version = src[0] & 15;
  if (version > 1) return -1;
  const int fecmax = version >= 1 ? 13 : 15;
  const uint8_t *code = src + 1;
  const uint8_t *data = code + index_count / 3;
  const uint8_t *end = src + size - 16;  // the aux table
  const uint8_t *aux_table = end;
  Fifos f;
  uint32_t next = 0, last = 0;
  for (size_t i = 0; i < index_count; i += 3) {
    const uint8_t ct = *code++;
    uint32_t a, b, c;
    if (ct < 0xf0) {
      const uint32_t *e = f.edge[(f.eo - 1 - (ct >> 4)) & 15];
      a = e[0];
      b = e[1];
      const int fec = ct & 15;
      if (fec < fecmax) {
        c = fec == 0 ? next : f.vert[(f.vo - 1 - fec) & 15];
        if (fec == 0) next++;
        f.push_vert(c, fec == 0);
      } else {
        if (fec != 15) c = last + uint32_t(fec - (fec ^ 3));
        else if (!get_index(data, end, last, c)) return -2;
        last = c;
        f.push_vert(c);
      }
      f.push_edge(c, b);
      f.push_edge(a, c);
    } else {
      uint8_t aux;
      int fea;
      const bool escape = ct >= 0xfe;  // aux code from the data; 15 = free index only here
      if (!escape) {
        aux = aux_table[ct & 15];
        fea = 0;
      } else {
        if (data >= end) return -2;
        aux = *data++;
        fea = ct == 0xfe ? 0 : 15;
        if (aux == 0) next = 0;  // reset: the stream restarts its vertex numbering
      }
      const int feb = aux >> 4, fec = aux & 15;
      a = fea == 0 ? next++ : 0;
      b = feb == 0 ? next++ : f.vert[(f.vo - feb) & 15];
      c = fec == 0 ? next++ : f.vert[(f.vo - fec) & 15];
      if (fea == 15) {
        if (!get_index(data, end, last, a)) return -2;
        last = a;
      }
      if (escape && feb == 15) {
        if (!get_index(data, end, last, b)) return -2;
        last = b;
      }
      if (escape && fec == 15) {
        if (!get_index(data, end, last, c)) return -2;
        last = c;
      }
      f.push_vert(a);
      f.push_vert(b, feb == 0 || (escape && feb == 15));
      f.push_vert(c, fec == 0 || (escape && fec == 15));
      f.push_edge(b, a);
      f.push_edge(c, b);
      f.push_edge(a, c);
    }
    out[i] = a;
    out[i + 1] = b;
    out[i + 2] = c;
  }
  if (data != end) return -3;
  return 0;
}

}  // extern "C"
