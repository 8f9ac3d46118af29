#include "fastx.h"

#include <zlib.h>

#include <algorithm>
#include <cstdint>
#include <cstring>

#include "error.h"
#include "zstd_io.h"

// The few entry points of liblzma (xz-utils 5.x) and libbzip2 (1.0.x) that
// query decoding uses, declared here from their stable public C APIs (the
// image ships the shared libraries without headers).
extern "C" {
struct zx_lzma_stream {
  const uint8_t* next_in;
  size_t avail_in;
  uint64_t total_in;
  uint8_t* next_out;
  size_t avail_out;
  uint64_t total_out;
  const void* allocator;
  void* internal;
  void* reserved_ptr[4];
  uint64_t reserved_int1, reserved_int2;
  size_t reserved_int3, reserved_int4;
  int reserved_enum1, reserved_enum2;
};
int lzma_stream_decoder(zx_lzma_stream* strm, uint64_t memlimit, uint32_t flags);
int lzma_code(zx_lzma_stream* strm, int action);
void lzma_end(zx_lzma_stream* strm);
struct zx_bz_stream {
  char* next_in;
  unsigned int avail_in;
  unsigned int total_in_lo32, total_in_hi32;
  char* next_out;
  unsigned int avail_out;
  unsigned int total_out_lo32, total_out_hi32;
  void* state;
  void* (*bzalloc)(void*, int, int);
  void (*bzfree)(void*, void*);
  void* opaque;
};
int BZ2_bzDecompressInit(zx_bz_stream* strm, int verbosity, int small);
int BZ2_bzDecompress(zx_bz_stream* strm);
int BZ2_bzDecompressEnd(zx_bz_stream* strm);
}

namespace zx {

namespace {

constexpr int kLzmaOk = 0, kLzmaStreamEnd = 1, kLzmaFinish = 3;
constexpr uint32_t kLzmaConcatenated = 0x08;
constexpr int kBzOk = 0, kBzStreamEnd = 4;

// .xz input (every stream of a concatenated file), as deko's xz decoder reads
// it for the reference parser (src/lib.rs:283-321).
std::vector<uint8_t> xz_decode_all(const std::vector<uint8_t>& raw, const std::string& path) {
  zx_lzma_stream zs;
  memset(&zs, 0, sizeof zs);
  check(lzma_stream_decoder(&zs, UINT64_MAX, kLzmaConcatenated) == kLzmaOk, kEFormat,
        "xz: cannot initialise decoder");
  std::vector<uint8_t> out, buf(1 << 20);
  zs.next_in = raw.data();
  zs.avail_in = raw.size();
  int rc = kLzmaOk;
  for (;;) {
    zs.next_out = buf.data();
    zs.avail_out = buf.size();
    rc = lzma_code(&zs, kLzmaFinish);
    out.insert(out.end(), buf.data(), buf.data() + (buf.size() - zs.avail_out));
    if (rc != kLzmaOk) break;
  }
  lzma_end(&zs);
  check(rc == kLzmaStreamEnd, kEFormat, ("corrupt or truncated xz input " + path).c_str());
  return out;
}

// .bz2 input, concatenated streams included.
std::vector<uint8_t> bz2_decode_all(const std::vector<uint8_t>& raw, const std::string& path) {
  std::vector<uint8_t> out, buf(1 << 20);
  size_t at = 0;
  while (at < raw.size()) {
    zx_bz_stream bs;
    memset(&bs, 0, sizeof bs);
    check(BZ2_bzDecompressInit(&bs, 0, 0) == kBzOk, kEFormat, "bzip2: cannot initialise decoder");
    bs.next_in = (char*)raw.data() + at;
    const size_t avail = std::min<size_t>(raw.size() - at, 0xFFFFFFFFu);
    bs.avail_in = (unsigned int)avail;
    int rc = kBzOk;
    for (;;) {
      bs.next_out = (char*)buf.data();
      bs.avail_out = (unsigned int)buf.size();
      rc = BZ2_bzDecompress(&bs);
      out.insert(out.end(), buf.data(), buf.data() + (buf.size() - bs.avail_out));
      if (rc != kBzOk) break;
      if (bs.avail_in == 0 && bs.avail_out != 0) break;  // input ended inside the stream
    }
    const size_t used = avail - bs.avail_in;
    BZ2_bzDecompressEnd(&bs);
    check(rc == kBzStreamEnd, kEFormat, ("corrupt or truncated bzip2 input " + path).c_str());
    at += used;
    // Trailing bytes that do not start another stream end the input.
    if (at + 3 > raw.size() || memcmp(raw.data() + at, "BZh", 3)) {
      check(at == raw.size(), kEFormat, ("unexpected data after bzip2 input " + path).c_str());
      break;
    }
  }
  return out;
}

std::vector<uint8_t> decoded_input(const std::string& path) {
  std::vector<uint8_t> raw = read_file_bytes(path);
  if (raw.size() >= 4 && raw[0] == 0x28 && raw[1] == 0xb5 && raw[2] == 0x2f && raw[3] == 0xfd)
    return zstd_decode_all(raw.data(), raw.size());
  if (raw.size() >= 2 && raw[0] == 0x1f && raw[1] == 0x8b) {
    z_stream zs;
    memset(&zs, 0, sizeof zs);
    check(inflateInit2(&zs, 15 + 32) == Z_OK, kEFormat, "gzip: cannot initialise decoder");
    std::vector<uint8_t> out;
    std::vector<uint8_t> buf(1 << 20);
    zs.next_in = raw.data();
    zs.avail_in = (uInt)raw.size();
    int rc = Z_OK;
    for (;;) {
      zs.next_out = buf.data();
      zs.avail_out = (uInt)buf.size();
      rc = inflate(&zs, Z_NO_FLUSH);
      if (rc != Z_OK && rc != Z_STREAM_END) break;
      out.insert(out.end(), buf.data(), buf.data() + (buf.size() - zs.avail_out));
      if (rc == Z_STREAM_END) {
        if (zs.avail_in == 0) break;
        // Concatenated gzip members.
        check(inflateReset(&zs) == Z_OK, kEFormat, "gzip: reset failed");
      }
    }
    inflateEnd(&zs);
    check(rc == Z_STREAM_END, kEFormat, ("corrupt or truncated gzip input " + path).c_str());
    return out;
  }
  if (raw.size() >= 6 && !memcmp(raw.data(), "\xfd" "7zXZ\0", 6)) return xz_decode_all(raw, path);
  if (raw.size() >= 3 && !memcmp(raw.data(), "BZh", 3)) return bz2_decode_all(raw, path);
  return raw;
}

inline const uint8_t* line_end(const uint8_t* p, const uint8_t* e) {
  const void* nl = memchr(p, '\n', (size_t)(e - p));
  return nl ? (const uint8_t*)nl : e;
}
inline const uint8_t* trim_cr(const uint8_t* a, const uint8_t* le) {
  return (le > a && le[-1] == '\r') ? le - 1 : le;
}
std::string header_name(const uint8_t* a, const uint8_t* e) {
  const uint8_t* p = a + 1;
  const uint8_t* q = p;
  while (q < e && *q != ' ' && *q != '\t' && *q != '\r') ++q;
  return std::string(p, q);
}

}  // namespace

void parse_fastx(const uint8_t* data, size_t len, RecordBatch& out, bool keep_names) {
  const uint8_t* p = data;
  const uint8_t* e = data + len;
  if (out.offsets.empty()) out.offsets.push_back(out.bases.size());
  while (p < e && (*p == '\n' || *p == '\r')) ++p;
  if (p == e) return;
  if (*p == '>') {
    while (p < e) {
      check_format(*p == '>', "malformed FASTA record");
      const uint8_t* he = line_end(p, e);
      if (keep_names) out.names.push_back(header_name(p, he));
      p = he < e ? he + 1 : e;
      while (p < e && *p != '>') {
        const uint8_t* le = line_end(p, e);
        const uint8_t* te = trim_cr(p, le);
        out.bases.insert(out.bases.end(), p, te);
        p = le < e ? le + 1 : e;
      }
      out.offsets.push_back(out.bases.size());
    }
    return;
  }
  check_format(*p == '@', "input is neither FASTA nor FASTQ");
  while (p < e) {
    if (*p == '\n' || *p == '\r') {
      ++p;
      continue;
    }
    check_format(*p == '@', "malformed FASTQ record");
    const uint8_t* he = line_end(p, e);
    check_format(he < e, "truncated FASTQ header");
    if (keep_names) out.names.push_back(header_name(p, he));
    p = he + 1;
    const uint8_t* se = line_end(p, e);
    const uint8_t* ste = trim_cr(p, se);
    check_format(se < e, "truncated FASTQ record");
    size_t seq_len = (size_t)(ste - p);
    out.bases.insert(out.bases.end(), p, ste);
    p = se + 1;
    check_format(p < e && *p == '+', "malformed FASTQ separator");
    const uint8_t* pe = line_end(p, e);
    check_format(pe < e, "truncated FASTQ record");
    p = pe + 1;
    const uint8_t* qe = line_end(p, e);
    const uint8_t* qte = trim_cr(p, qe);
    check_format((size_t)(qte - p) == seq_len, "truncated FASTQ quality");
    p = qe < e ? qe + 1 : e;
    out.offsets.push_back(out.bases.size());
  }
}

namespace {

inline bool ascii_ws(uint8_t c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\f' || c == '\v';
}

// Well-formed UTF-8 (no overlong forms, no surrogates, at most U+10FFFF).
bool valid_utf8(const uint8_t* p, const uint8_t* e) {
  while (p < e) {
    const uint8_t c = *p;
    int n;
    uint32_t cp;
    if (c < 0x80) {
      ++p;
      continue;
    } else if (c >= 0xc2 && c <= 0xdf) {
      n = 1, cp = c & 0x1f;
    } else if (c >= 0xe0 && c <= 0xef) {
      n = 2, cp = c & 0x0f;
    } else if (c >= 0xf0 && c <= 0xf4) {
      n = 3, cp = c & 0x07;
    } else {
      return false;
    }
    if (e - p <= n) return false;
    for (int i = 1; i <= n; ++i) {
      if ((p[i] & 0xc0) != 0x80) return false;
      cp = (cp << 6) | (p[i] & 0x3f);
    }
    if ((n == 2 && (cp < 0x800 || (cp >= 0xd800 && cp <= 0xdfff))) ||
        (n == 3 && (cp < 0x10000 || cp > 0x10ffff)))
      return false;
    p += n + 1;
  }
  return true;
}

// Line reader over a byte buffer: [a, b) is the line without its '\n'.
struct Lines {
  const uint8_t* p;
  const uint8_t* e;
  bool next(const uint8_t*& a, const uint8_t*& b) {
    if (p >= e) return false;
    a = p;
    b = line_end(p, e);
    p = b < e ? b + 1 : e;
    return true;
  }
};

}  // namespace

void parse_named_records(const uint8_t* data, size_t len, RecordBatch& out) {
  if (out.offsets.empty()) out.offsets.push_back(out.bases.size());
  Lines lines{data, data + len};
  const uint8_t *a, *b;
  int fastq = -1;
  bool open = false;  // a FASTA record is being read
  auto identifier = [&](const char* kind) {
    const uint8_t* q = a + 1;
    while (q < b && !ascii_ws(*q)) ++q;
    check_format(q > a + 1, (std::string("empty ") + kind + " identifier").c_str());
    check_format(valid_utf8(a + 1, q), (std::string("invalid ") + kind + " identifier").c_str());
    out.names.emplace_back(a + 1, q);
  };
  auto no_whitespace = [&](const char* msg) {
    for (const uint8_t* q = a; q < b; ++q) check_format(!ascii_ws(*q), msg);
  };
  auto trim_line_end = [&] {
    while (b > a && (b[-1] == '\n' || b[-1] == '\r')) --b;
  };
  while (lines.next(a, b)) {
    while (b > a && ascii_ws(b[-1])) --b;
    if (a == b) continue;
    if (fastq == 1 || (fastq == -1 && *a == '@')) {
      fastq = 1;
      check_format(*a == '@', "expected FASTQ identifier");
      identifier("FASTQ");
      const size_t start = out.bases.size();
      for (;;) {
        check_format(lines.next(a, b), "truncated FASTQ sequence");
        trim_line_end();
        if (b > a && *a == '+') break;
        no_whitespace("whitespace inside FASTQ sequence");
        out.bases.insert(out.bases.end(), a, b);
      }
      const size_t seq = out.bases.size() - start;
      size_t qualities = 0;
      while (qualities < seq) {
        check_format(lines.next(a, b), "truncated FASTQ quality");
        trim_line_end();
        qualities += (size_t)(b - a);
        check_format(qualities <= seq, "FASTQ sequence and quality lengths differ");
      }
      out.offsets.push_back(out.bases.size());
      continue;
    }
    fastq = 0;
    if (*a == '>') {
      if (open) out.offsets.push_back(out.bases.size());
      identifier("FASTA");
      open = true;
    } else {
      check_format(open, "--records requires FASTA or FASTQ");
      no_whitespace("whitespace inside FASTA sequence");
      out.bases.insert(out.bases.end(), a, b);
    }
  }
  if (open) out.offsets.push_back(out.bases.size());
  check_format(out.offsets.size() > 1, "no FASTA/FASTQ records");
}

RecordBatch read_named_records(const std::string& path) {
  std::vector<uint8_t> data = decoded_input(path);
  RecordBatch batch;
  batch.bases.reserve(data.size());
  parse_named_records(data.data(), data.size(), batch);
  return batch;
}

RecordBatch read_fastx(const std::string& path, bool keep_names) {
  std::vector<uint8_t> data = decoded_input(path);
  RecordBatch batch;
  batch.bases.reserve(data.size());
  parse_fastx(data.data(), data.size(), batch, keep_names);
  if (batch.offsets.empty()) batch.offsets.push_back(0);
  return batch;
}

}  // namespace zx
