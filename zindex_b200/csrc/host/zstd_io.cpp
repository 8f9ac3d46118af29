#include "zstd_io.h"

#include <atomic>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <thread>

#include "error.h"

// libzstd public API (zstd.h is not installed here; libzstd.so.1 is).
extern "C" {
typedef struct ZSTD_DCtx_s ZSTD_DCtx;
typedef struct ZSTD_CCtx_s ZSTD_CCtx;
typedef struct {
  const void* src;
  size_t size;
  size_t pos;
} ZSTD_inBuffer;
typedef struct {
  void* dst;
  size_t size;
  size_t pos;
} ZSTD_outBuffer;
ZSTD_DCtx* ZSTD_createDCtx(void);
size_t ZSTD_freeDCtx(ZSTD_DCtx*);
size_t ZSTD_decompressDCtx(ZSTD_DCtx*, void*, size_t, const void*, size_t);
size_t ZSTD_decompressStream(ZSTD_DCtx*, ZSTD_outBuffer*, ZSTD_inBuffer*);
size_t ZSTD_DCtx_reset(ZSTD_DCtx*, int);
unsigned long long ZSTD_getFrameContentSize(const void*, size_t);
size_t ZSTD_findFrameCompressedSize(const void*, size_t);
ZSTD_CCtx* ZSTD_createCCtx(void);
size_t ZSTD_freeCCtx(ZSTD_CCtx*);
size_t ZSTD_CCtx_setParameter(ZSTD_CCtx*, int, int);
size_t ZSTD_compress2(ZSTD_CCtx*, void*, size_t, const void*, size_t);
size_t ZSTD_compressBound(size_t);
unsigned ZSTD_isError(size_t);
const char* ZSTD_getErrorName(size_t);
}

namespace zx {
namespace {

constexpr size_t kChunk = 4u << 20;
constexpr size_t kHeader = 40;
constexpr uint32_t kSkip = 0x184D2A50u;
constexpr int kCompressionLevel = 100;  // ZSTD_c_compressionLevel
constexpr int kChecksumFlag = 201;      // ZSTD_c_checksumFlag
constexpr int kResetSession = 1;        // ZSTD_reset_session_only

uint64_t le64(const uint8_t* p) {
  uint64_t v = 0;
  for (int i = 7; i >= 0; --i) v = (v << 8) | p[i];
  return v;
}
uint32_t le32(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
void put64(std::vector<uint8_t>& v, uint64_t x) {
  for (int i = 0; i < 8; ++i) v.push_back((uint8_t)(x >> (8 * i)));
}
uint64_t fnv1a(const uint8_t* p, size_t n) {
  uint64_t h = 0xcbf29ce484222325ull;
  for (size_t i = 0; i < n; ++i) h = (h ^ p[i]) * 0x100000001b3ull;
  return h;
}
bool is_zstd(const uint8_t* p, size_t n) {
  return n >= 4 && p[0] == 0x28 && p[1] == 0xb5 && p[2] == 0x2f && p[3] == 0xfd;
}
void zcheck(size_t r, const char* what) {
  if (ZSTD_isError(r)) raise(kEFormat, std::string(what) + ": " + ZSTD_getErrorName(r));
}

// Streams `in` into the sink; returns decoded byte count.
template <class Sink>
size_t stream_decode(const uint8_t* in, size_t len, Sink&& sink) {
  ZSTD_DCtx* d = ZSTD_createDCtx();
  std::vector<uint8_t> buf(1 << 20);
  ZSTD_inBuffer ib{in, len, 0};
  size_t total = 0, last = 0;
  try {
    for (;;) {
      ZSTD_outBuffer ob{buf.data(), buf.size(), 0};
      last = ZSTD_decompressStream(d, &ob, &ib);
      zcheck(last, "zstd stream");
      if (ob.pos) sink(buf.data(), ob.pos);
      total += ob.pos;
      if (ib.pos == ib.size && ob.pos < ob.size) break;
    }
  } catch (...) {
    ZSTD_freeDCtx(d);
    throw;
  }
  ZSTD_freeDCtx(d);
  check_format(last == 0, "truncated zstd stream");
  return total;
}

struct FrameInfo {
  uint64_t compressed, compressed_len, raw, raw_len;
};

// Seek table of a framed bank (bank_io.rs:114-197). Empty when absent.
std::vector<FrameInfo> seek_table(const std::vector<uint8_t>& f, size_t raw_total) {
  std::vector<FrameInfo> frames;
  size_t length = f.size();
  if (length < 16 || memcmp(&f[length - 16], "ZORSEEK1", 8) != 0) return frames;
  uint64_t len = le64(&f[length - 8]);
  check_format(len >= 40 && len <= (64u << 20) && (len - 40) % 32 == 0 && len + 8 <= length,
               "invalid bank seek table length");
  size_t start = length - len - 8;
  check_format(le32(&f[start]) == kSkip && le32(&f[start + 4]) == len,
               "invalid skippable bank index");
  const uint8_t* t = &f[start + 8];
  check_format(memcmp(t, "ZORFRM1\0", 8) == 0 && memcmp(t + len - 16, "ZORSEEK1", 8) == 0 &&
                   le64(t + len - 8) == len,
               "invalid bank seek table tag");
  check_format(le64(t + len - 24) == fnv1a(t, len - 24), "bank seek table checksum mismatch");
  uint64_t count = le64(t + 8);
  check_format(count == (len - 40) / 32 && count != 0 && count <= raw_total,
               "invalid bank frame count");
  uint64_t compressed = 0, raw = 0;
  for (uint64_t i = 0; i < count; ++i) {
    const uint8_t* e = t + 16 + 32 * i;
    FrameInfo fr{le64(e), le64(e + 8), le64(e + 16), le64(e + 24)};
    check_format(fr.compressed == compressed && fr.raw == raw && fr.raw_len >= 1 &&
                     fr.raw_len <= kChunk && fr.compressed_len > 0 &&
                     fr.compressed_len <= fr.raw_len + fr.raw_len / 128 + 1024,
                 "invalid bank frame geometry");
    compressed += fr.compressed_len;
    raw += fr.raw_len;
    check_format(compressed <= start && raw <= raw_total, "bank frame exceeds payload");
    frames.push_back(fr);
  }
  check_format(compressed == start && raw == raw_total && frames[0].raw_len >= kHeader,
               "incomplete bank frame coverage");
  return frames;
}

}  // namespace

std::vector<uint8_t> read_file_bytes(const std::string& path) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) raise(kEIo, "cannot open " + path + ": " + strerror(errno));
  fseek(f, 0, SEEK_END);
  long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  std::vector<uint8_t> data(n > 0 ? (size_t)n : 0);
  size_t got = data.empty() ? 0 : fread(data.data(), 1, data.size(), f);
  fclose(f);
  if (got != data.size()) raise(kEIo, "short read of " + path);
  return data;
}

void write_file_bytes(const std::string& path, const void* data, size_t len) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) raise(kEIo, "cannot create " + path + ": " + strerror(errno));
  size_t put = len ? fwrite(data, 1, len, f) : 0;
  int rc = fclose(f);
  if (put != len || rc != 0) raise(kEIo, "short write of " + path);
}

std::vector<uint8_t> zstd_decode_all(const uint8_t* data, size_t len) {
  if (!is_zstd(data, len)) return std::vector<uint8_t>(data, data + len);
  std::vector<uint8_t> out;
  stream_decode(data, len, [&](const uint8_t* p, size_t n) { out.insert(out.end(), p, p + n); });
  return out;
}

void read_bank_stream(const std::string& path, uint8_t header[40], uint8_t* payload,
                      size_t payload_len, int threads) {
  std::vector<uint8_t> file = read_file_bytes(path);
  const size_t raw_total = payload_len + kHeader;
  std::vector<FrameInfo> frames = seek_table(file, raw_total);
  if (frames.size() <= 1) {
    // Stream decode (legacy single stream or one frame).
    size_t at = 0;
    bool extra = false;
    auto sink = [&](const uint8_t* p, size_t n) {
      for (size_t i = 0; i < n;) {
        if (at < kHeader) {
          size_t take = std::min(n - i, kHeader - at);
          memcpy(header + at, p + i, take);
          at += take;
          i += take;
        } else if (at - kHeader < payload_len) {
          size_t take = std::min(n - i, payload_len - (at - kHeader));
          memcpy(payload + (at - kHeader), p + i, take);
          at += take;
          i += take;
        } else {
          extra = true;
          return;
        }
      }
    };
    if (is_zstd(file.data(), file.size()))
      stream_decode(file.data(), file.size(), sink);
    else
      sink(file.data(), file.size());
    check_format(at == raw_total, "short bank data");
    check_format(!extra, "unexpected bank data");
    return;
  }
  // Parallel frames straight into the destination (bank_io.rs:235-292).
  std::atomic<size_t> next{0};
  std::atomic<bool> failed{false};
  std::string error;
  std::vector<uint8_t> first(frames[0].raw_len);
  auto worker = [&]() {
    ZSTD_DCtx* d = ZSTD_createDCtx();
    for (size_t i; !failed && (i = next.fetch_add(1)) < frames.size();) {
      const FrameInfo& fr = frames[i];
      const uint8_t* src = file.data() + fr.compressed;
      bool ok = ZSTD_findFrameCompressedSize(src, fr.compressed_len) == fr.compressed_len &&
                ZSTD_getFrameContentSize(src, fr.compressed_len) == fr.raw_len;
      uint8_t* dst = i == 0 ? first.data() : payload + (fr.raw - kHeader);
      if (ok) {
        size_t r = ZSTD_decompressDCtx(d, dst, fr.raw_len, src, fr.compressed_len);
        ok = !ZSTD_isError(r) && r == fr.raw_len;
      }
      if (!ok && !failed.exchange(true)) error = "corrupt bank frame in " + path;
    }
    ZSTD_freeDCtx(d);
  };
  int n = std::max(1, std::min<int>(threads, (int)frames.size()));
  std::vector<std::thread> pool;
  for (int t = 1; t < n; ++t) pool.emplace_back(worker);
  worker();
  for (auto& th : pool) th.join();
  if (failed) raise(kEFormat, error);
  memcpy(header, first.data(), kHeader);
  memcpy(payload, first.data() + kHeader, frames[0].raw_len - kHeader);
}

FramedWriter::FramedWriter(const std::string& path, int level) : path_(path), level_(level) {
  file_ = fopen(path.c_str(), "wb");
  if (!file_) raise(kEIo, "cannot create " + path + ": " + strerror(errno));
  cctx_ = ZSTD_createCCtx();
  ZSTD_CCtx_setParameter((ZSTD_CCtx*)cctx_, kCompressionLevel, level_);
  ZSTD_CCtx_setParameter((ZSTD_CCtx*)cctx_, kChecksumFlag, 1);
  pending_.reserve(kChunk);
}

FramedWriter::~FramedWriter() {
  if (file_) fclose((FILE*)file_);
  if (cctx_) ZSTD_freeCCtx((ZSTD_CCtx*)cctx_);
}

void FramedWriter::flush_frame() {
  if (pending_.empty()) return;
  encoded_.resize(ZSTD_compressBound(pending_.size()));
  size_t r = ZSTD_compress2((ZSTD_CCtx*)cctx_, encoded_.data(), encoded_.size(), pending_.data(),
                            pending_.size());
  zcheck(r, "zstd compress");
  if (fwrite(encoded_.data(), 1, r, (FILE*)file_) != r) raise(kEIo, "short write of " + path_);
  frames_.push_back(Frame{compressed_, r, raw_, pending_.size()});
  compressed_ += r;
  raw_ += pending_.size();
  pending_.clear();
}

void FramedWriter::write(const void* data, size_t len) {
  const uint8_t* p = (const uint8_t*)data;
  while (len) {
    size_t take = std::min(len, kChunk - pending_.size());
    pending_.insert(pending_.end(), p, p + take);
    p += take;
    len -= take;
    if (pending_.size() == kChunk) flush_frame();
  }
}

void FramedWriter::finish() {
  flush_frame();
  check(!frames_.empty(), kEInval, "empty bank stream");
  std::vector<uint8_t> table;
  table.insert(table.end(), (const uint8_t*)"ZORFRM1\0", (const uint8_t*)"ZORFRM1\0" + 8);
  put64(table, frames_.size());
  for (auto& f : frames_) {
    put64(table, f.compressed);
    put64(table, f.compressed_len);
    put64(table, f.raw);
    put64(table, f.raw_len);
  }
  put64(table, fnv1a(table.data(), table.size()));
  table.insert(table.end(), (const uint8_t*)"ZORSEEK1", (const uint8_t*)"ZORSEEK1" + 8);
  uint64_t len = table.size() + 8;
  put64(table, len);
  uint8_t skip[8];
  for (int i = 0; i < 4; ++i) skip[i] = (uint8_t)(kSkip >> (8 * i));
  for (int i = 0; i < 4; ++i) skip[4 + i] = (uint8_t)(len >> (8 * i));
  FILE* f = (FILE*)file_;
  bool ok = fwrite(skip, 1, 8, f) == 8 && fwrite(table.data(), 1, table.size(), f) == table.size();
  ok = (fclose(f) == 0) && ok;
  file_ = nullptr;
  if (!ok) raise(kEIo, "short write of " + path_);
}

void write_zstd_file(const std::string& path, const void* data, size_t len, int level) {
  ZSTD_CCtx* c = ZSTD_createCCtx();
  ZSTD_CCtx_setParameter(c, kCompressionLevel, level);
  ZSTD_CCtx_setParameter(c, kChecksumFlag, 1);
  std::vector<uint8_t> out(ZSTD_compressBound(len));
  size_t r = ZSTD_compress2(c, out.data(), out.size(), data, len);
  ZSTD_freeCCtx(c);
  zcheck(r, "zstd compress");
  write_file_bytes(path, out.data(), r);
}

}  // namespace zx
