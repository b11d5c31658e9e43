// dcd.cu -- DCD trajectory files: host-side header and layout parsing,
// threaded pread into pinned memory, unit-cell decoding, and the device
// decode kernel (record markers, byte order, atom selection, length scale).
//
// Follows the record structure and error behaviour of warp-md's DcdReader
// (crates/traj-io/src/dcd.rs): header detection 833-870, open 45-95, frames
// 207-291 and 433-498, unit cells 978-1101.  The reference reads a frame at a
// time through a 1 MiB BufReader and converts on the CPU; here every frame of
// a batch is one contiguous pread and the conversion runs on the GPU.
#include "dcd.h"

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstring>

#include "device_util.cuh"

namespace wmd {

namespace {

constexpr int kDecodeThreads = 256;
constexpr int kDecodeAtoms = 1024;  // atoms per work item of the decode kernel

DcdError make_err(int kind, const char* msg) {
  DcdError e;
  e.kind = kind;
  e.msg = msg;
  return e;
}

DcdError io_eof() { return make_err(kDcdIo, "failed to fill whole buffer"); }

bool pread_full(int fd, void* dst, int64_t len, int64_t off) {
  char* p = static_cast<char*>(dst);
  while (len > 0) {
    const ssize_t r = ::pread(fd, p, (size_t)std::min<int64_t>(len, int64_t(1) << 30), (off_t)off);
    if (r < 0 && errno == EINTR) continue;
    if (r <= 0) return false;
    p += r;
    off += r;
    len -= r;
  }
  return true;
}

uint32_t bswap32(uint32_t v) { return __builtin_bswap32(v); }
uint64_t bswap64(uint64_t v) { return __builtin_bswap64(v); }

// Record marker at pos (caller checked the bounds).
DcdError marker_at(const DcdFile& f, int64_t pos, uint64_t* out) {
  uint8_t b[8];
  if (pos + f.marker > f.file_size || !pread_full(f.fd, b, f.marker, pos)) return io_eof();
  if (f.marker == 4) {
    uint32_t v;
    std::memcpy(&v, b, 4);
    *out = f.big ? bswap32(v) : v;
  } else {
    uint64_t v;
    std::memcpy(&v, b, 8);
    *out = f.big ? bswap64(v) : v;
  }
  return {};
}

int32_t i32_of(const uint8_t* p, bool big) {
  uint32_t v;
  std::memcpy(&v, p, 4);
  return (int32_t)(big ? bswap32(v) : v);
}

bool header_len_ok(uint64_t v) { return v == 84 || v == 164; }

// One frame from pos as the reference's read_frame walks it.  *eof is set
// when the trajectory ends cleanly before a coordinate record; otherwise
// *next is the first byte after the frame and *cell its unit-cell payload.
DcdError walk_frame(const DcdFile& f, int64_t pos, int64_t* next, int32_t* cell, bool* eof) {
  const int64_t M = f.marker, rec = 4 * f.n_atoms;
  *eof = false;
  *cell = 0;
  uint64_t len = 0, end = 0;
  if (pos + M > f.file_size) {
    *eof = true;
    return {};
  }
  if (DcdError e = marker_at(f, pos, &len)) return e;
  pos += M;
  if ((int64_t)len != rec && (len == 24 || len == 48)) {
    if (pos + (int64_t)len > f.file_size) return io_eof();
    pos += (int64_t)len;
    if (DcdError e = marker_at(f, pos, &end)) return e;
    pos += M;
    if (end != len) return make_err(kDcdParse, "unitcell record length mismatch");
    *cell = (int32_t)len;
    if (pos + M > f.file_size) {
      *eof = true;
      return {};
    }
    if (DcdError e = marker_at(f, pos, &len)) return e;
    pos += M;
  }
  if ((int64_t)len != rec) return make_err(kDcdParse, "unexpected DCD coordinate record length");
  for (int axis = 0; axis < 3; ++axis) {
    if (axis > 0) {
      if (DcdError e = marker_at(f, pos, &len)) return e;
      pos += M;
      if ((int64_t)len != rec) return make_err(kDcdParse, "unexpected float record length");
    }
    if (pos + rec > f.file_size) return io_eof();
    pos += rec;
    if (DcdError e = marker_at(f, pos, &end)) return e;
    pos += M;
    if (end != len) return make_err(kDcdParse, "float record length mismatch");
  }
  *next = pos;
  return {};
}

double to_radians(double v) { return v * (3.14159265358979323846 / 180.0); }

// unitcell_angle_to_radians (dcd.rs:1095-1101): cosines when |v| <= 1
double angle_to_radians(double v) {
  if (std::fabs(v) <= 1.0) return std::acos(std::min(std::max(v, -1.0), 1.0));
  return to_radians(v);
}

// box_from_values (dcd.rs:1024-1093)
int box_from_values(const double v[6], bool charmm, float scale, float m[9]) {
  double a, b, c, al, be, ga;
  if (charmm) {
    a = v[0]; b = v[2]; c = v[5]; al = v[4]; be = v[3]; ga = v[1];
  } else {
    a = v[0]; b = v[1]; c = v[2]; al = v[3]; be = v[4]; ga = v[5];
  }
  a *= (double)scale;
  b *= (double)scale;
  c *= (double)scale;
  for (int i = 0; i < 9; ++i) m[i] = 0.f;
  const double min_len = 1e-6;
  if (!std::isfinite(a) || !std::isfinite(b) || !std::isfinite(c) || a <= min_len || b <= min_len || c <= min_len)
    return 0;
  const double ar = angle_to_radians(al), br = angle_to_radians(be), gr = angle_to_radians(ga);
  if (!std::isfinite(ar) || !std::isfinite(br) || !std::isfinite(gr)) return 0;
  const double ninety = 1.57079632679489661923, tol = 1e-3;
  if (std::fabs(ar - ninety) < tol && std::fabs(br - ninety) < tol && std::fabs(gr - ninety) < tol) {
    m[0] = (float)a;
    m[4] = (float)b;
    m[8] = (float)c;
    return 1;
  }
  const double ca = std::cos(ar), cb = std::cos(br), cg = std::cos(gr), sg = std::sin(gr);
  if (std::fabs(sg) < 1e-8) return 0;
  const double cx = c * cb, cy = c * (ca - cb * cg) / sg;
  const double cz2 = c * c - cx * cx - cy * cy;
  if (!std::isfinite(cz2) || cz2 <= 0.0) return 0;
  m[0] = (float)a;
  m[3] = (float)(b * cg);
  m[4] = (float)(b * sg);
  m[6] = (float)cx;
  m[7] = (float)cy;
  m[8] = (float)std::sqrt(cz2);
  return 2;
}

// ---------------------------------------------------------------------------
// device decode
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t ld_bytes_u32(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

__device__ __forceinline__ uint32_t dev_bswap(uint32_t v) { return __byte_perm(v, 0, 0x0123); }

__device__ __forceinline__ uint64_t dev_marker(const uint8_t* p, int marker, bool big) {
  const uint32_t w0 = ld_bytes_u32(p);
  if (marker == 4) return big ? dev_bswap(w0) : w0;
  const uint32_t w1 = ld_bytes_u32(p + 4);
  return big ? ((uint64_t)dev_bswap(w0) << 32) | dev_bswap(w1) : ((uint64_t)w1 << 32) | w0;
}

template <bool ALIGNED>
__device__ __forceinline__ float ld_coord(const uint8_t* p, bool big, float scale) {
  uint32_t w = ALIGNED ? __ldg(reinterpret_cast<const uint32_t*>(p)) : ld_bytes_u32(p);
  if (big) w = dev_bswap(w);
  const float v = __uint_as_float(w);
  return scale == 1.f ? v : __fmul_rn(v, scale);
}

// out[f][i] = (x, y, z) of atom sel[i] (or i) of batch frame f.  Work items
// are (frame, block of kDecodeAtoms output atoms).  In the uniform layout the
// first item of each frame also checks the frame's record markers against
// the layout assumed for the file; the indexed layout was checked on the
// host.
template <bool ALIGNED>
__global__ void __launch_bounds__(kDecodeThreads) dcd_decode_kernel(DcdDecode d) {
  const int64_t tiles = (d.n_out + kDecodeAtoms - 1) / kDecodeAtoms;
  const int64_t items = tiles * d.n_frames;
  const int64_t M = d.marker, rec = 4 * d.n_atoms;
  for (int64_t it = blockIdx.x; it < items; it += gridDim.x) {
    const int64_t f = it / tiles, t = it - f * tiles;
    const int64_t xo =
        d.xoff ? d.xoff[f] : d.data_start + (d.first + f) * d.stride + (d.cell ? 2 * M + d.cell : 0);
    const uint8_t* X = d.raw + (xo - d.raw_off);
    if (!d.xoff && t == 0 && threadIdx.x < 8) {
      const int k = threadIdx.x;
      const uint8_t* p = nullptr;
      int64_t want = rec;
      if (k < 6) {
        p = X + (k >> 1) * (2 * M + rec) + (k & 1) * (M + rec);
      } else if (d.cell) {
        p = X - 2 * M - d.cell + (k == 7 ? M + d.cell : 0);
        want = d.cell;
      }
      if (p && dev_marker(p, d.marker, d.big) != (uint64_t)want) atomicOr(d.status, kStatusBadRecord);
    }
    const uint8_t* px = X + M;
    const uint8_t* py = px + rec + 2 * M;
    const uint8_t* pz = py + rec + 2 * M;
    float* o = d.out + (size_t)f * d.n_out * 3;
    const int64_t i_end = min(d.n_out, (t + 1) * kDecodeAtoms);
    for (int64_t i = t * kDecodeAtoms + threadIdx.x; i < i_end; i += kDecodeThreads) {
      int64_t a = i;
      if (d.sel) {
        a = d.sel[i];
        if (a >= d.n_atoms) {
          atomicOr(d.status, kStatusBadIndex);
          continue;
        }
      }
      o[3 * i + 0] = ld_coord<ALIGNED>(px + 4 * a, d.big, d.scale);
      o[3 * i + 1] = ld_coord<ALIGNED>(py + 4 * a, d.big, d.scale);
      o[3 * i + 2] = ld_coord<ALIGNED>(pz + 4 * a, d.big, d.scale);
    }
  }
}

}  // namespace

DcdError dcd_open(const char* path, float length_scale, DcdFile* f) {
  *f = DcdFile();
  f->length_scale = length_scale;
  f->fd = ::open(path, O_RDONLY | O_CLOEXEC);
  if (f->fd < 0) return make_err(kDcdIo, std::strerror(errno));
  struct stat st;
  if (fstat(f->fd, &st) != 0) return make_err(kDcdIo, std::strerror(errno));
  f->file_size = (int64_t)st.st_size;
  // detect_header_marker: 8-byte markers first, then 4-byte
  uint8_t head[8];
  if (f->file_size < 8 || !pread_full(f->fd, head, 8, 0)) return io_eof();
  uint64_t v8;
  uint32_t v4;
  std::memcpy(&v8, head, 8);
  std::memcpy(&v4, head, 4);
  uint64_t hlen = 0;
  if (header_len_ok(v8)) {
    f->marker = 8, f->big = false, hlen = v8;
  } else if (header_len_ok(bswap64(v8))) {
    f->marker = 8, f->big = true, hlen = bswap64(v8);
  } else if (header_len_ok(v4)) {
    f->marker = 4, f->big = false, hlen = v4;
  } else if (header_len_ok(bswap32(v4))) {
    f->marker = 4, f->big = true, hlen = bswap32(v4);
  } else {
    return make_err(kDcdUnsupported, "unsupported DCD record marker");
  }
  const int64_t M = f->marker;
  int64_t pos = M;
  uint8_t header[164];
  if (pos + (int64_t)hlen > f->file_size || !pread_full(f->fd, header, (int64_t)hlen, pos)) return io_eof();
  pos += (int64_t)hlen;
  uint64_t len = 0;
  if (DcdError e = marker_at(*f, pos, &len)) return e;
  pos += M;
  if (len != hlen) return make_err(kDcdParse, "DCD header record length mismatch");
  if (std::memcmp(header, "CORD", 4) == 0) {
    const int32_t n = i32_of(header + 4, f->big);
    f->header_frames = n > 0 ? n : 0;
  }
  f->charmm = i32_of(header + 80, f->big) > 0;  // parse_unitcell_layout: CHARMM version slot
  // title record
  if (DcdError e = marker_at(*f, pos, &len)) return e;
  pos += M;
  if (pos + (int64_t)len > f->file_size) return io_eof();
  pos += (int64_t)len;
  uint64_t end = 0;
  if (DcdError e = marker_at(*f, pos, &end)) return e;
  pos += M;
  if (end != len) return make_err(kDcdParse, "record length mismatch");
  // natoms record
  if (DcdError e = marker_at(*f, pos, &len)) return e;
  pos += M;
  if (len != 4) return make_err(kDcdParse, "unexpected natoms record length");
  uint8_t nb[4];
  if (pos + 4 > f->file_size || !pread_full(f->fd, nb, 4, pos)) return io_eof();
  pos += 4;
  const int32_t natoms = i32_of(nb, f->big);
  if (DcdError e = marker_at(*f, pos, &end)) return e;
  pos += M;
  if (end != 4) return make_err(kDcdParse, "natoms record length mismatch");
  if (natoms <= 0) return make_err(kDcdParse, "invalid natoms");
  f->n_atoms = natoms;
  f->data_start = pos;

  // Layout from the first frame; the rest of the file is assumed to repeat it
  // (the decode kernel checks every frame's markers, and a file that differs
  // is indexed frame by frame).
  int64_t next = 0;
  int32_t cell = 0;
  bool eof = false;
  DcdError e0 = walk_frame(*f, pos, &next, &cell, &eof);
  if (e0 || eof) {
    f->n_frames = 0;
    f->stride = 1;
    f->end = e0;
    return {};
  }
  f->stride = next - pos;
  f->cell = cell;
  const int64_t n_full = (f->file_size - f->data_start) / f->stride;
  // the last whole frame must repeat the layout and what follows must end
  // cleanly; anything else is resolved by walking every frame
  int64_t nl = 0;
  int32_t cl = 0;
  DcdError el = walk_frame(*f, f->data_start + (n_full - 1) * f->stride, &nl, &cl, &eof);
  bool uniform = !el && !eof && cl == cell && nl == f->data_start + n_full * f->stride;
  if (uniform) {
    DcdError et = walk_frame(*f, nl, &next, &cell, &eof);
    uniform = !et && eof;
  }
  if (!uniform) return dcd_index(f);
  f->n_frames = n_full;
  return {};
}

DcdError dcd_index(DcdFile* f) {
  f->indexed = true;
  f->fbeg.clear();
  f->fcell.clear();
  f->end = DcdError();
  int64_t pos = f->data_start;
  for (;;) {
    int64_t next = 0;
    int32_t cell = 0;
    bool eof = false;
    DcdError e = walk_frame(*f, pos, &next, &cell, &eof);
    if (e) {
      f->end = e;
      break;
    }
    if (eof) break;
    f->fbeg.push_back(pos);
    f->fcell.push_back(cell);
    pos = next;
  }
  f->n_frames = (int64_t)f->fbeg.size();
  f->fbeg.push_back(pos);
  return {};
}

void dcd_close(DcdFile* f) {
  if (f->fd >= 0) ::close(f->fd);
  f->fd = -1;
}

ReadPool::ReadPool(int threads) {
  // a thread that cannot be started leaves a smaller pool (the caller always
  // takes parts itself), never a half-built object
  try {
    workers_.reserve((size_t)std::max(threads - 1, 0));
    for (int t = 1; t < threads; ++t) workers_.emplace_back([this] { work(); });
  } catch (...) {
  }
}

ReadPool::~ReadPool() {
  {
    std::lock_guard<std::mutex> g(m_);
    stop_ = true;
  }
  wake_.notify_all();
  for (auto& t : workers_) t.join();
}

bool ReadPool::take(int* i) {  // m_ held
  if (!fn_ || next_ >= parts_) return false;
  *i = next_++;
  return true;
}

void ReadPool::work() {
  std::unique_lock<std::mutex> lk(m_);
  for (;;) {
    int i;
    wake_.wait(lk, [&] { return stop_ || (fn_ && next_ < parts_); });
    if (stop_) return;
    while (take(&i)) {
      const std::function<void(int)>* fn = fn_;
      lk.unlock();
      (*fn)(i);
      lk.lock();
      if (--pending_ == 0) done_.notify_all();
    }
  }
}

void ReadPool::run(int parts, const std::function<void(int)>& fn) {
  if (parts <= 0) return;
  std::unique_lock<std::mutex> lk(m_);
  fn_ = &fn;
  next_ = 0;
  parts_ = parts;
  pending_ = parts;
  wake_.notify_all();
  int i;
  while (take(&i)) {
    lk.unlock();
    fn(i);
    lk.lock();
    --pending_;
  }
  done_.wait(lk, [&] { return pending_ == 0; });
  fn_ = nullptr;
  parts_ = 0;
}

DcdError dcd_pread(const DcdFile& f, ReadPool& pool, void* dst, int64_t off, int64_t len) {
  if (off < 0 || off + len > f.file_size) return io_eof();
  const int64_t part = int64_t(2) << 20;
  const int parts = (int)std::max<int64_t>(1, std::min<int64_t>((len + part - 1) / part, 4096));
  if (parts == 1 || pool.size() == 1) return pread_full(f.fd, dst, len, off) ? DcdError() : io_eof();
  const int64_t step = ((len + parts - 1) / parts + 4095) & ~int64_t(4095);
  std::vector<char> ok((size_t)parts, 1);
  pool.run(parts, [&](int p) {
    const int64_t a = p * step, b = std::min(len, a + step);
    if (a < b) ok[p] = pread_full(f.fd, static_cast<char*>(dst) + a, b - a, off + a);
  });
  for (char c : ok)
    if (!c) return io_eof();
  return {};
}

int dcd_box(const DcdFile& f, const uint8_t* payload, int64_t len, float m[9]) {
  double v[6];
  for (int i = 0; i < 6; ++i) {
    if (len == 24) {
      uint32_t w;
      std::memcpy(&w, payload + 4 * i, 4);
      if (f.big) w = bswap32(w);
      float x;
      std::memcpy(&x, &w, 4);
      v[i] = x;
    } else {
      uint64_t w;
      std::memcpy(&w, payload + 8 * i, 8);
      if (f.big) w = bswap64(w);
      std::memcpy(&v[i], &w, 8);
    }
  }
  const int k = box_from_values(v, f.charmm, f.length_scale, m);
  if (k) return k;
  // the reference retries the other layout (producer variants)
  return box_from_values(v, !f.charmm, f.length_scale, m);
}

cudaError_t launch_dcd_decode(const DcdDecode& d, int sm_count, cudaStream_t s) {
  if (d.n_frames == 0 || d.n_out == 0) return cudaSuccess;
  const int64_t items = ((d.n_out + kDecodeAtoms - 1) / kDecodeAtoms) * d.n_frames;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(items, (int64_t)sm_count * 8));
  if (d.aligned) dcd_decode_kernel<true><<<grid, kDecodeThreads, 0, s>>>(d);
  else dcd_decode_kernel<false><<<grid, kDecodeThreads, 0, s>>>(d);
  return cudaGetLastError();
}

}  // namespace wmd
