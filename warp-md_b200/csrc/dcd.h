// dcd.h -- DCD trajectory files (internal; the C ABI is in
// include/warpmd_rmsd.h).
//
// The host reads the header and the layout of the first frame, then moves raw
// frame bytes (pread into pinned memory, several threads) to the device,
// where dcd_decode_kernel checks every record marker, swaps big-endian words,
// gathers the selected atoms, applies the length scale and writes packed
// float32 xyz.  Unit cells are decoded on the host from the same pinned bytes.
#pragma once

#include <cuda_runtime.h>

#include <condition_variable>
#include <cstdint>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace wmd {

// Error classes of the reference reader (TrajError::Io / Parse / Unsupported).
enum DcdErrKind { kDcdOk = 0, kDcdIo = 1, kDcdParse = 2, kDcdUnsupported = 3 };

struct DcdError {
  int kind = kDcdOk;
  std::string msg;
  explicit operator bool() const { return kind != kDcdOk; }
};

struct DcdFile {
  int fd = -1;
  bool big = false;      // big-endian records
  int marker = 4;        // record marker bytes (4 or 8)
  int64_t n_atoms = 0;
  int64_t header_frames = 0;  // the header's frame count when > 0, else 0
  bool charmm = false;        // unit cells as [A, gamma, B, beta, alpha, C]
  float length_scale = 1.f;
  int64_t data_start = 0, file_size = 0;
  // Frames [0, n_frames) are readable.  Uniform layout: frame f starts at
  // data_start + f * stride and carries a unit-cell record of `cell` payload
  // bytes (0 = none).  Indexed layout (a file whose frames differ): fbeg[f]
  // (n_frames + 1 entries) and fcell[f].
  int64_t n_frames = 0;
  bool indexed = false;
  int64_t stride = 0, cell = 0;
  std::vector<int64_t> fbeg;
  std::vector<int32_t> fcell;
  DcdError end;  // raised by a read that continues past n_frames (none: clean end of file)

  int64_t frame_begin(int64_t f) const { return indexed ? fbeg[f] : data_start + f * stride; }
  int64_t frame_cell(int64_t f) const { return indexed ? fcell[f] : cell; }
  // file offset of the X record's leading marker
  int64_t frame_x(int64_t f) const {
    const int64_t c = frame_cell(f);
    return frame_begin(f) + (c ? 2 * marker + c : 0);
  }
};

// Persistent threads for the parallel preads of a batch; the calling thread
// takes parts too.
class ReadPool {
 public:
  explicit ReadPool(int threads);
  ~ReadPool();
  int size() const { return (int)workers_.size() + 1; }
  // fn(i) for every i in [0, parts), spread over the pool; returns when all are done
  void run(int parts, const std::function<void(int)>& fn);

 private:
  void work();
  bool take(int* i);
  std::vector<std::thread> workers_;
  std::mutex m_;
  std::condition_variable wake_, done_;
  const std::function<void(int)>* fn_ = nullptr;
  int next_ = 0, parts_ = 0, pending_ = 0;
  bool stop_ = false;
};

// Opens and parses the header (dcd.rs:45-95) and the frame layout.
DcdError dcd_open(const char* path, float length_scale, DcdFile* f);
void dcd_close(DcdFile* f);
// Walks every frame's record markers from data_start as the reference's
// sequential reader does (dcd.rs:207-291) and switches to the indexed layout;
// the first damaged frame ends the readable range and becomes `end`.
DcdError dcd_index(DcdFile* f);
// pread of [off, off + len) into dst in parts of a few MiB spread over the pool.
DcdError dcd_pread(const DcdFile& f, ReadPool& pool, void* dst, int64_t off, int64_t len);
// Box of one frame from its unit-cell payload (read_unitcell_with_len +
// box_from_values, dcd.rs:978-1093): returns 0 none, 1 orthorhombic,
// 2 triclinic; m = the box vectors a, b, c as rows.
int dcd_box(const DcdFile& f, const uint8_t* payload, int64_t len, float m[9]);

struct DcdDecode {
  const uint8_t* raw = nullptr;  // device copy of the file from offset raw_off
  int64_t raw_off = 0;
  int64_t first = 0;             // first frame of the batch
  int64_t n_frames = 0;
  const int64_t* xoff = nullptr; // indexed layout: X-marker file offset per batch frame (device)
  int64_t data_start = 0, stride = 0, cell = 0;  // uniform layout
  int64_t n_atoms = 0;
  int marker = 4;
  bool big = false;
  bool aligned = true;           // every record payload starts on a 4-byte boundary
  float scale = 1.f;
  const uint32_t* sel = nullptr; // device; null = atoms 0 .. n_out-1
  int64_t n_out = 0;
  float* out = nullptr;          // [n_frames][n_out][3]
  int* status = nullptr;
};

cudaError_t launch_dcd_decode(const DcdDecode& d, int sm_count, cudaStream_t s);

}  // namespace wmd
