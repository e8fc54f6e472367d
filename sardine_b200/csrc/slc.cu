// Sentinel-1 SLC measurement TIFF ingest (slc_reader.rs): the classic-TIFF
// IFD checks of parse_ifd (268-465) and burst reads of read_burst_raw
// (532-583), feeding device memory directly.
//
// A read into device memory streams the rows through pinned host buffers:
// four threads pread 32 MB chunks in parallel, each filling one of its two
// buffers while the other's host-to-device copy runs on the context's
// stream, so the file reads and the copies overlap.
// Big-endian files (never written for Sentinel-1) are byte-swapped on the
// device after the copy.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>

#include "runtime.cuh"

constexpr int kSlcThreads = 4;                 // reader threads of a device read
constexpr uint64_t kSlcChunk = 32ull << 20;     // bytes per pinned buffer (two per thread)

struct sd_slc_reader {
  int fd = -1;
  uint32_t width = 0, height = 0;
  bool le = true;
  uint64_t base = 0, row_bytes = 0;
  std::string path;
  int device = -1;                              // pinned buffers below belong to this device's reads
  void *pin[2 * kSlcThreads] = {nullptr};
  cudaEvent_t ev[2 * kSlcThreads] = {nullptr};
};

namespace sd {
namespace {

constexpr uint16_t kTagWidth = 256, kTagLength = 257, kTagBps = 258, kTagCompression = 259,
                   kTagStripOffsets = 273, kTagSpp = 277, kTagRowsPerStrip = 278, kTagSampleFormat = 339;

uint16_t rd16(const uint8_t *b, bool le) { return le ? (uint16_t)(b[0] | b[1] << 8) : (uint16_t)(b[1] | b[0] << 8); }
uint32_t rd32(const uint8_t *b, bool le) {
  return le ? (uint32_t)b[0] | (uint32_t)b[1] << 8 | (uint32_t)b[2] << 16 | (uint32_t)b[3] << 24
            : (uint32_t)b[3] | (uint32_t)b[2] << 8 | (uint32_t)b[1] << 16 | (uint32_t)b[0] << 24;
}

// pread of exactly n bytes; false on a short read or error (read_exact).
bool pread_all(int fd, void *dst, size_t n, uint64_t off) {
  uint8_t *p = (uint8_t *)dst;
  while (n > 0) {
    const ssize_t k = ::pread(fd, p, n, (off_t)off);
    if (k < 0 && errno == EINTR) continue;
    if (k <= 0) return false;
    p += k;
    n -= (size_t)k;
    off += (uint64_t)k;
  }
  return true;
}

__global__ void k_swap16(uint16_t *d, uint64_t n) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d[i] = (uint16_t)((d[i] >> 8) | (d[i] << 8));
}

int io_error(sd_ctx *ctx, const std::string &path) {
  return set_error(ctx, SD_ERR_SLC_IO, "I/O error: %s: %s", path.c_str(), errno ? std::strerror(errno) : "short read");
}

}  // namespace
}  // namespace sd

using namespace sd;

extern "C" int sd_slc_open(sd_ctx *ctx, const char *path, sd_slc_reader **out) {
  if (!ctx || !path || !out) return SD_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  sd_slc_reader r;
  r.path = path;
  errno = 0;
  r.fd = ::open(path, O_RDONLY | O_CLOEXEC);
  if (r.fd < 0) return io_error(ctx, r.path);
  struct Fd {
    int &fd;
    ~Fd() {
      if (fd >= 0) ::close(fd);
    }
  } guard{r.fd};
  uint8_t h[8];
  errno = 0;
  if (!pread_all(r.fd, h, 8, 0)) return io_error(ctx, r.path);
  bool le;
  if (h[0] == 'I' && h[1] == 'I') le = true;
  else if (h[0] == 'M' && h[1] == 'M') le = false;
  else return set_error(ctx, SD_ERR_SLC_NOT_TIFF, "not a classic TIFF (bad byte-order marker or magic=0)");
  const uint16_t magic = rd16(h + 2, le);
  if (magic == 43)
    return set_error(ctx, SD_ERR_SLC_BIGTIFF, "BigTIFF (magic=43) is not supported; only classic TIFF (magic=42) is accepted");
  if (magic != 42) return set_error(ctx, SD_ERR_SLC_NOT_TIFF, "not a classic TIFF (bad byte-order marker or magic=%u)", magic);
  const uint64_t ifd = rd32(h + 4, le);
  uint8_t nb[2];
  errno = 0;
  if (!pread_all(r.fd, nb, 2, ifd)) return io_error(ctx, r.path);
  const uint32_t n = rd16(nb, le);
  std::vector<uint8_t> e((size_t)n * 12);
  if (n > 0 && !pread_all(r.fd, e.data(), e.size(), ifd + 2)) return io_error(ctx, r.path);

  // the tags parse_ifd reads; SHORT/LONG scalars inline, StripOffsets kept raw
  bool has[8] = {false};
  uint32_t val[8] = {0};
  uint16_t so_type = 0;
  uint32_t so_count = 0, so_value = 0;
  bool has_so = false;
  const uint16_t tags[7] = {kTagWidth, kTagLength, kTagBps, kTagCompression, kTagRowsPerStrip, kTagSpp,
                            kTagSampleFormat};
  for (uint32_t k = 0; k < n; ++k) {
    const uint8_t *p = e.data() + 12 * k;
    const uint16_t tag = rd16(p, le), typ = rd16(p + 2, le);
    const uint32_t count = rd32(p + 4, le);
    if (tag == kTagStripOffsets) {
      so_type = typ;
      so_count = count;
      so_value = rd32(p + 8, le);
      has_so = true;
      continue;
    }
    for (int t = 0; t < 7; ++t)
      if (tag == tags[t]) {
        // entry_scalar: SHORT from the first 2 bytes, LONG from 4, else none
        if (typ == 3) {
          has[t] = true;
          val[t] = rd16(p + 8, le);
        } else if (typ == 4) {
          has[t] = true;
          val[t] = rd32(p + 8, le);
        } else {
          has[t] = false;
        }
      }
  }
  // the order of parse_ifd's checks
  const int order[6] = {0, 1, 2, 3, 4, 6};  // width, length, bps, compression, rows/strip, sample format
  for (int t : order)
    if (!has[t]) return set_error(ctx, SD_ERR_SLC_MISSING_TAG, "required TIFF tag %u is absent from the IFD", tags[t]);
  if (!has_so) return set_error(ctx, SD_ERR_SLC_MISSING_TAG, "required TIFF tag %u is absent from the IFD", kTagStripOffsets);
  const uint32_t width = val[0], height = val[1];
  const uint16_t bps = (uint16_t)val[2], comp = (uint16_t)val[3], sfmt = (uint16_t)val[6];
  const uint32_t rps = val[4];
  const uint16_t spp = has[5] ? (uint16_t)val[5] : 1;
  if (comp != 1) return set_error(ctx, SD_ERR_SLC_UNSUPPORTED_FORMAT, "unsupported TIFF format: Compression=%u (expected 1=None)", comp);
  if (sfmt != 5) return set_error(ctx, SD_ERR_SLC_UNSUPPORTED_FORMAT, "unsupported TIFF format: SampleFormat=%u (expected 5=CInt)", sfmt);
  if (bps != 32)
    return set_error(ctx, SD_ERR_SLC_UNSUPPORTED_FORMAT, "unsupported TIFF format: BitsPerSample=%u (expected 32 for CInt16)", bps);
  if (rps != 1) return set_error(ctx, SD_ERR_SLC_UNSUPPORTED_FORMAT, "unsupported TIFF format: RowsPerStrip=%u (expected 1)", rps);
  if (spp != 1)
    return set_error(ctx, SD_ERR_SLC_UNSUPPORTED_FORMAT, "unsupported TIFF format: SamplesPerPixel=%u (expected 1 for CInt16)", spp);
  if (so_count != height)
    return set_error(ctx, SD_ERR_SLC_UNSUPPORTED_FORMAT, "unsupported TIFF format: strip count (%u) != image height (%u)",
                     so_count, height);
  if (height == 0) return set_error(ctx, SD_ERR_SLC_UNSUPPORTED_FORMAT, "unsupported TIFF format: image height 0");
  const uint64_t row_bytes = (uint64_t)width * 4;
  uint64_t base, last;
  if (so_count == 1) {
    base = last = so_value;
  } else {
    if (so_type != 3 && so_type != 4)
      return set_error(ctx, SD_ERR_SLC_UNSUPPORTED_FORMAT,
                       "unsupported TIFF format: StripOffsets field type %u is not SHORT(3) or LONG(4)", so_type);
    const uint64_t each = so_type == 3 ? 2 : 4;
    uint8_t b[4];
    errno = 0;
    if (!pread_all(r.fd, b, each, so_value)) return io_error(ctx, r.path);
    base = so_type == 3 ? rd16(b, le) : rd32(b, le);
    if (!pread_all(r.fd, b, each, so_value + (uint64_t)(so_count - 1) * each)) return io_error(ctx, r.path);
    last = so_type == 3 ? rd16(b, le) : rd32(b, le);
  }
  const uint64_t expected = base + (uint64_t)(height - 1) * row_bytes;
  if (last != expected)
    return set_error(ctx, SD_ERR_SLC_NON_CONTIGUOUS_STRIPS,
                     "strip offsets not contiguous (strip[0]=%llu, strip[%u-1]=%llu, expected=%llu); direct-seek "
                     "reader cannot be used",
                     (unsigned long long)base, so_count, (unsigned long long)last, (unsigned long long)expected);
  r.width = width;
  r.height = height;
  r.le = le;
  r.base = base;
  r.row_bytes = row_bytes;
  sd_slc_reader *res = new sd_slc_reader(r);
  r.fd = -1;  // now owned by res
  *out = res;
  return SD_OK;
}

extern "C" int sd_slc_dims(const sd_slc_reader *r, uint32_t *width, uint32_t *height, int32_t *little_endian) {
  if (!r) return SD_ERR_INVALID_ARGUMENT;
  if (width) *width = r->width;
  if (height) *height = r->height;
  if (little_endian) *little_endian = r->le ? 1 : 0;
  return SD_OK;
}

extern "C" void sd_slc_close(sd_slc_reader *r) {
  if (!r) return;
  if (r->device >= 0) cudaSetDevice(r->device);
  for (int k = 0; k < 2 * kSlcThreads; ++k) {
    if (r->ev[k]) {
      cudaEventSynchronize(r->ev[k]);
      cudaEventDestroy(r->ev[k]);
    }
    if (r->pin[k]) cudaFreeHost(r->pin[k]);
  }
  if (r->fd >= 0) ::close(r->fd);
  delete r;
}

extern "C" int sd_slc_read_burst_raw(sd_ctx *ctx, sd_slc_reader *r, uint64_t first_line, uint64_t line_count,
                                     int16_t *out) {
  SD_STAGE("read_burst");
  if (!ctx || !r) return SD_ERR_INVALID_ARGUMENT;
  if (first_line > r->height || line_count > (uint64_t)r->height - first_line)
    return set_error(ctx, SD_ERR_SLC_LINE_OUT_OF_BOUNDS, "line range [%llu, %llu) is out of image bounds [0, %u)",
                     (unsigned long long)first_line, (unsigned long long)(first_line + line_count), r->height);
  if (line_count == 0) return SD_OK;
  if (!out) return set_error(ctx, SD_ERR_INVALID_ARGUMENT, "null output");
  const uint64_t bytes = line_count * r->row_bytes, off = r->base + first_line * r->row_bytes;
  if (!is_device_ptr(out)) {  // host destination: one read
    errno = 0;
    if (!pread_all(r->fd, out, bytes, off)) return io_error(ctx, r->path);
    if (!r->le) {
      uint16_t *q = (uint16_t *)out;
      for (uint64_t i = 0; i < bytes / 2; ++i) q[i] = (uint16_t)((q[i] >> 8) | (q[i] << 8));
    }
    return SD_OK;
  }
  SD_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  if (r->device != ctx->device) {  // pinned buffers and events, kept for the reader's later reads
    for (int k = 0; k < 2 * kSlcThreads; ++k) {
      if (r->ev[k]) cudaEventDestroy(r->ev[k]);
      if (r->pin[k]) cudaFreeHost(r->pin[k]);
      r->pin[k] = nullptr;
      r->ev[k] = nullptr;
    }
    r->device = ctx->device;
    for (int k = 0; k < 2 * kSlcThreads; ++k) {
      SD_CUDA(ctx, cudaHostAlloc(&r->pin[k], kSlcChunk, cudaHostAllocDefault));
      SD_CUDA(ctx, cudaEventCreateWithFlags(&r->ev[k], cudaEventDisableTiming));
    }
  }
  // Chunk c goes to thread c % T and, within it, alternates between the
  // thread's two buffers: each thread reads one chunk while its previous
  // chunk's copy runs; the threads' reads proceed in parallel.
  const uint64_t n_chunks = (bytes + kSlcChunk - 1) / kSlcChunk;
  const int nt = (int)std::min<uint64_t>(kSlcThreads, n_chunks);
  std::atomic<int> fail{0};
  std::mutex err_mu;
  int err_code = SD_OK;
  std::string err_msg;
  auto worker = [&](int t) {
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
      fail = 1;
      return;
    }
    bool used[2] = {false, false};
    int b = 0;
    for (uint64_t c = (uint64_t)t; c < n_chunks && !fail.load(); c += (uint64_t)nt) {
      const int k = 2 * t + b;
      const uint64_t o = c * kSlcChunk, n = std::min(kSlcChunk, bytes - o);
      cudaError_t ce = cudaSuccess;
      if (used[b]) ce = cudaEventSynchronize(r->ev[k]);  // its previous copy has left the buffer
      bool ok = ce == cudaSuccess;
      int saved = 0;
      if (ok) {
        errno = 0;
        ok = pread_all(r->fd, r->pin[k], n, off + o);
        saved = errno;
        if (ok) ce = cudaMemcpyAsync((uint8_t *)out + o, r->pin[k], n, cudaMemcpyHostToDevice, s);
        if (ok && ce == cudaSuccess) ce = cudaEventRecord(r->ev[k], s);
      }
      if (!ok || ce != cudaSuccess) {
        std::lock_guard<std::mutex> g(err_mu);
        if (err_code == SD_OK) {
          err_code = !ok && ce == cudaSuccess ? SD_ERR_SLC_IO : SD_ERR_CUDA;
          err_msg = err_code == SD_ERR_SLC_IO ? (saved ? std::strerror(saved) : "short read") : cudaGetErrorString(ce);
        }
        fail = 1;
        return;
      }
      used[b] = true;
      b ^= 1;
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) th.emplace_back(worker, t);
  worker(0);
  for (auto &x : th) x.join();
  if (err_code != SD_OK) {
    cudaStreamSynchronize(s);
    return set_error(ctx, err_code, "%s%s: %s", err_code == SD_ERR_SLC_IO ? "I/O error: " : "", r->path.c_str(),
                     err_msg.c_str());
  }
  if (!r->le) {
    const uint64_t nh = bytes / 2;
    SD_TIMED_BEGIN(ctx, "k_swap16");
    k_swap16<<<(unsigned)((nh + 255) / 256), 256, 0, s>>>((uint16_t *)out, nh);
    SD_LAUNCHED(ctx);
  }
  return sync(ctx);
}
