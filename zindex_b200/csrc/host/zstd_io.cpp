#include "zstd_io.h"

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <atomic>
#include <cerrno>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
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
// tail: the file's last len + 8 bytes (the skippable frame holding the
// table), which start at file offset `start`.
std::vector<FrameInfo> seek_table(const std::vector<uint8_t>& tail, uint64_t start,
                                  size_t raw_total) {
  std::vector<FrameInfo> frames;
  const uint64_t len = tail.size() - 8;
  check_format(len >= 40 && (len - 40) % 32 == 0, "invalid bank seek table length");
  check_format(le32(&tail[0]) == kSkip && le32(&tail[4]) == len, "invalid skippable bank index");
  const uint8_t* t = &tail[8];
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

namespace {

struct Fd {
  int fd = -1;
  ~Fd() {
    if (fd >= 0) close(fd);
  }
};

void pread_full(int fd, uint8_t* dst, size_t n, uint64_t off, const std::string& path) {
  while (n) {
    ssize_t r = pread(fd, dst, n, (off_t)off);
    if (r < 0 && errno == EINTR) continue;
    if (r <= 0) raise(kEIo, "short read of " + path);
    dst += r;
    n -= (size_t)r;
    off += (uint64_t)r;
  }
}

}  // namespace

void stream_bank(const std::string& path, uint8_t header[40], uint64_t payload_len,
                 uint64_t piece_bytes, uint8_t* const* ring, int slots, int threads,
                 PieceSink& sink) {
  // A frame then touches at most two pieces, and a frame that straddles
  // pieces c and c+1 can always be written while piece c is being filled.
  check(slots >= 3 && piece_bytes >= kChunk, kEInval,
        "bank streaming needs three ring slots of at least one 4 MiB frame");
  const uint64_t raw_total = payload_len + kHeader;
  const uint64_t pieces = (payload_len + piece_bytes - 1) / piece_bytes;
  auto piece_len = [&](uint64_t c) { return std::min(piece_bytes, payload_len - c * piece_bytes); };
  Fd f;
  f.fd = open(path.c_str(), O_RDONLY);
  if (f.fd < 0) raise(kEIo, "cannot open " + path + ": " + strerror(errno));
  struct stat st;
  if (fstat(f.fd, &st) != 0) raise(kEIo, "cannot stat " + path);
  const uint64_t file_len = (uint64_t)st.st_size;
  // The seek table is the file's tail: read only that, then frames on demand.
  std::vector<FrameInfo> frames;
  if (file_len >= 16) {
    uint8_t tail16[16];
    pread_full(f.fd, tail16, 16, file_len - 16, path);
    if (!memcmp(tail16, "ZORSEEK1", 8)) {
      const uint64_t len = le64(tail16 + 8);
      check_format(len >= 40 && len <= (64u << 20) && len + 8 <= file_len,
                   "invalid bank seek table length");
      std::vector<uint8_t> tail(len + 8);
      pread_full(f.fd, tail.data(), tail.size(), file_len - len - 8, path);
      frames = seek_table(tail, file_len - len - 8, raw_total);
    }
  }
  if (frames.size() <= 1) {
    // Legacy single stream (or one frame): decoded in order on this thread.
    std::vector<uint8_t> file = read_file_bytes(path);
    uint64_t at = 0, c = 0, fill = 0;
    bool extra = false;
    auto emit = [&](const uint8_t* p, size_t n) {
      for (size_t i = 0; i < n;) {
        if (at < kHeader) {
          size_t take = std::min<uint64_t>(n - i, kHeader - at);
          memcpy(header + at, p + i, take);
          at += take;
          i += take;
        } else if (at - kHeader < payload_len) {
          if (fill == 0 && c >= (uint64_t)slots) sink.drain((int)(c % slots));
          size_t take = std::min<uint64_t>(n - i, piece_len(c) - fill);
          memcpy(ring[c % slots] + fill, p + i, take);
          fill += take;
          at += take;
          i += take;
          if (fill == piece_len(c)) {
            sink.consume((int)(c % slots), c * piece_bytes, fill);
            ++c;
            fill = 0;
          }
        } else {
          extra = true;
          return;
        }
      }
    };
    if (is_zstd(file.data(), file.size()))
      stream_decode(file.data(), file.size(), emit);
    else
      emit(file.data(), file.size());
    check_format(at == raw_total, "short bank data");
    check_format(!extra, "unexpected bank data");
    for (int sl = 0; sl < slots; ++sl) sink.drain(sl);
    return;
  }
  // Frames (bank_io.rs:235-292) are decoded by the workers in frame order
  // into the ring; piece c lives in slot c % slots and may be written once
  // the consumer has released piece c - slots. The calling thread hands
  // every complete piece to the sink in order.
  std::mutex mu;
  std::condition_variable cv_filled, cv_free;
  std::vector<uint64_t> filled(pieces, 0);
  uint64_t released = 0;  // pieces [0, released) no longer occupy their slots
  bool failed = false;
  std::string error;
  std::atomic<size_t> next{0};
  auto fail = [&](const std::string& msg) {
    std::lock_guard<std::mutex> lock(mu);
    if (!failed) error = msg;
    failed = true;
    cv_filled.notify_all();
    cv_free.notify_all();
  };
  auto worker = [&]() {
    ZSTD_DCtx* d = ZSTD_createDCtx();
    std::vector<uint8_t> src, tmp;
    try {
      for (size_t i; (i = next.fetch_add(1)) < frames.size();) {
        {
          std::lock_guard<std::mutex> lock(mu);
          if (failed) break;
        }
        const FrameInfo& fr = frames[i];
        // Payload bytes of this frame (frame 0 also carries the header).
        const uint64_t p0 = fr.raw < kHeader ? 0 : fr.raw - kHeader;
        const uint64_t p1 = fr.raw + fr.raw_len - kHeader;
        const uint64_t c0 = p0 / piece_bytes, c1 = p1 > p0 ? (p1 - 1) / piece_bytes : c0;
        src.resize(fr.compressed_len);
        pread_full(f.fd, src.data(), src.size(), fr.compressed, path);
        bool ok = ZSTD_findFrameCompressedSize(src.data(), src.size()) == fr.compressed_len &&
                  ZSTD_getFrameContentSize(src.data(), src.size()) == fr.raw_len;
        if (!ok) {
          fail("corrupt bank frame in " + path);
          break;
        }
        {
          std::unique_lock<std::mutex> lock(mu);
          cv_free.wait(lock, [&] { return failed || (p1 <= p0) || c1 < released + slots; });
          if (failed) break;
        }
        const bool direct = i != 0 && c0 == c1;
        uint8_t* dst;
        if (direct) {
          dst = ring[c0 % slots] + (p0 - c0 * piece_bytes);
        } else {
          tmp.resize(fr.raw_len);
          dst = tmp.data();
        }
        size_t r = ZSTD_decompressDCtx(d, dst, fr.raw_len, src.data(), src.size());
        if (ZSTD_isError(r) || r != fr.raw_len) {
          fail("corrupt bank frame in " + path);
          break;
        }
        const uint8_t* body = dst;
        if (i == 0) {
          memcpy(header, dst, kHeader);
          body = dst + kHeader;
        }
        if (!direct)
          for (uint64_t c = c0; p1 > p0 && c <= c1; ++c) {
            const uint64_t a = std::max(p0, c * piece_bytes);
            const uint64_t b = std::min(p1, c * piece_bytes + piece_len(c));
            memcpy(ring[c % slots] + (a - c * piece_bytes), body + (a - p0), b - a);
          }
        std::lock_guard<std::mutex> lock(mu);
        for (uint64_t c = c0; p1 > p0 && c <= c1; ++c) {
          const uint64_t a = std::max(p0, c * piece_bytes);
          const uint64_t b = std::min(p1, c * piece_bytes + piece_len(c));
          filled[c] += b - a;
        }
        cv_filled.notify_all();
      }
    } catch (const std::exception& e) {
      fail(e.what());
    }
    ZSTD_freeDCtx(d);
  };
  const int n = std::max(1, std::min<int>(threads, (int)frames.size()));
  std::vector<std::thread> pool;
  for (int t = 0; t < n; ++t) pool.emplace_back(worker);
  try {
    for (uint64_t c = 0; c < pieces; ++c) {
      {
        std::unique_lock<std::mutex> lock(mu);
        cv_filled.wait(lock, [&] { return failed || filled[c] == piece_len(c); });
        if (failed) break;
      }
      sink.consume((int)(c % slots), c * piece_bytes, piece_len(c));
      // One piece in flight: once the previous piece is consumed its slot
      // is free for piece c - 1 + slots.
      if (c >= 1) {
        sink.drain((int)((c - 1) % slots));
        std::lock_guard<std::mutex> lock(mu);
        released = c;
        cv_free.notify_all();
      }
    }
  } catch (const std::exception& e) {
    fail(e.what());
  }
  for (auto& th : pool) th.join();
  for (int sl = 0; sl < slots; ++sl) sink.drain(sl);
  if (failed) raise(kEFormat, error);
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
