// Bank and recovery-file byte streams. Bank files are independently
// decodable zstd frames of 4 MiB raw plus a skippable seek table
// (src/power_merge/bank_io.rs:11-16, 28-112, 114-292); the recovery file and
// legacy banks are one zstd stream (src/lib.rs:374-398).
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace zx {

std::vector<uint8_t> read_file_bytes(const std::string& path);
void write_file_bytes(const std::string& path, const void* data, size_t len);

// Decode a whole zstd stream (any number of frames, skippable frames ignored);
// raw input without the zstd magic is returned unchanged.
std::vector<uint8_t> zstd_decode_all(const uint8_t* data, size_t len);

// Decoded bank stream = 40-byte header + payload. Frames are decoded in
// parallel (threads) straight into `payload` (payload_len bytes). When the
// file has no seek table it is stream-decoded. Throws zx::Error on any
// mismatch, corruption or trailing data.
void read_bank_stream(const std::string& path, uint8_t header[40], uint8_t* payload,
                      size_t payload_len, int threads);

// Writer of the framed format with its seek table.
class FramedWriter {
 public:
  FramedWriter(const std::string& path, int level);
  ~FramedWriter();
  void write(const void* data, size_t len);
  void finish();

 private:
  struct Frame {
    uint64_t compressed, compressed_len, raw, raw_len;
  };
  void flush_frame();
  std::string path_;
  int level_;
  void* file_ = nullptr;
  std::vector<uint8_t> pending_, encoded_;
  std::vector<Frame> frames_;
  uint64_t compressed_ = 0, raw_ = 0;
  void* cctx_ = nullptr;
};

// One zstd frame (with checksum) of `data` written to `path`.
void write_zstd_file(const std::string& path, const void* data, size_t len, int level);

}  // namespace zx
