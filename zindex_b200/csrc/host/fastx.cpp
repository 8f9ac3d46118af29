#include "fastx.h"

#include <zlib.h>

#include <cstring>

#include "error.h"
#include "zstd_io.h"

namespace zx {

namespace {

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
  if ((raw.size() >= 6 && !memcmp(raw.data(), "\xfd" "7zXZ\0", 6)) ||
      (raw.size() >= 3 && !memcmp(raw.data(), "BZh", 3)))
    raise(kEUnsupported, "xz and bzip2 query inputs are not supported: " + path);
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

RecordBatch read_fastx(const std::string& path, bool keep_names) {
  std::vector<uint8_t> data = decoded_input(path);
  RecordBatch batch;
  batch.bases.reserve(data.size());
  parse_fastx(data.data(), data.size(), batch, keep_names);
  if (batch.offsets.empty()) batch.offsets.push_back(0);
  return batch;
}

}  // namespace zx
