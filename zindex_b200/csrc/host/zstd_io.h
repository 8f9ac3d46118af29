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

// Consumer of a streamed bank payload (see stream_bank).
class PieceSink {
 public:
  virtual ~PieceSink() = default;
  // Payload bytes [offset, offset + len) are complete in ring slot `slot`:
  // start consuming them (for example an asynchronous copy to the device).
  virtual void consume(int slot, uint64_t offset, uint64_t len) = 0;
  // Returns once the slot's last consumed piece is no longer read (its
  // buffer may be rewritten); a no-op for a slot with nothing in flight.
  virtual void drain(int slot) = 0;
};

// Decoded bank stream = 40-byte header + payload (payload_len bytes). The
// header goes to `header`; the payload is handed to `sink` in order, in
// pieces of piece_bytes (at least 4 MiB, one frame; the last piece may be
// shorter) through a ring of `slots` (>= 3) caller-owned buffers of
// piece_bytes each (piece c in slot c % slots). Frames are read with pread and decoded by `threads` workers in
// frame order straight into the ring, so reading, decoding and the sink's
// consumption overlap; the file is never held whole in memory. When the file
// has no seek table it is stream-decoded on the calling thread. Throws
// zx::Error on any mismatch, corruption or trailing data; every slot is
// drained before it returns or throws.
void stream_bank(const std::string& path, uint8_t header[40], uint64_t payload_len,
                 uint64_t piece_bytes, uint8_t* const* ring, int slots, int threads,
                 PieceSink& sink);

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
