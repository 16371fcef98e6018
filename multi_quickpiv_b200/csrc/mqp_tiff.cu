// Time-lapse ingest: a multi-page TIFF reader (host code) and a frame source
// that reads frames ahead into a ring of pinned host buffers for the serving
// path.  The reference reads its 2D+t and 3D+t stacks with LIBTIFF
// (README.md:55-68); this reader covers the baseline layouts such stacks use:
// classic little- or big-endian TIFF, one sample per pixel, strips or tiles,
// no compression or PackBits, unsigned/signed 8/16/32-bit integers and
// 32/64-bit floats.  Pages are returned in Julia's array order: a page of
// height H and width W becomes the column-major H x W array whose element
// (y, x) sits at y + H x (dimension 1 = image rows), and consecutive pages
// stack along dimension 3.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <stdint.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <condition_variable>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "mqp.h"

namespace {

struct Page {
  int64_t width = 0, height = 0;
  int bits = 0, format = 1, compression = 1;
  bool tiled = false;
  int64_t rows_per_strip = 0, tile_w = 0, tile_h = 0;
  std::vector<uint64_t> offsets, counts;
};

}  // namespace

struct mqp_tiff {
  int fd = -1;
  const uint8_t* map = nullptr;
  size_t size = 0;
  bool big_endian = false;
  std::vector<Page> pages;
  std::string last_error;
};

namespace {

int tiff_fail(mqp_tiff* t, int code, const std::string& msg) {
  if (t) t->last_error = msg;
  return code;
}

uint16_t rd16(const mqp_tiff* t, size_t o) {
  const uint8_t* p = t->map + o;
  return t->big_endian ? (uint16_t)((p[0] << 8) | p[1]) : (uint16_t)(p[0] | (p[1] << 8));
}
uint32_t rd32(const mqp_tiff* t, size_t o) {
  const uint8_t* p = t->map + o;
  return t->big_endian ? ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3]
                       : (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

// The values of one IFD entry (SHORT or LONG, inline or at an offset).
bool entry_values(const mqp_tiff* t, size_t e, std::vector<uint64_t>& out, std::string& err) {
  const uint16_t type = rd16(t, e + 2);
  const uint32_t count = rd32(t, e + 4);
  const int sz = type == 3 ? 2 : (type == 4 ? 4 : (type == 1 ? 1 : 0));
  if (!sz) {
    err = "unsupported TIFF field type " + std::to_string(type);
    return false;
  }
  size_t at = e + 8;
  if ((uint64_t)count * sz > 4) at = rd32(t, e + 8);
  if (at + (uint64_t)count * sz > t->size) {
    err = "TIFF field outside the file";
    return false;
  }
  out.resize(count);
  for (uint32_t i = 0; i < count; ++i)
    out[i] = sz == 2 ? rd16(t, at + 2 * i) : (sz == 4 ? rd32(t, at + 4 * i) : t->map[at + i]);
  return true;
}

int parse(mqp_tiff* t) {
  if (t->size < 8) return tiff_fail(t, MQP_ERR_INVALID, "not a TIFF file (too short)");
  if (t->map[0] == 'I' && t->map[1] == 'I') t->big_endian = false;
  else if (t->map[0] == 'M' && t->map[1] == 'M') t->big_endian = true;
  else return tiff_fail(t, MQP_ERR_INVALID, "not a TIFF file (byte order mark)");
  const uint16_t magic = rd16(t, 2);
  if (magic == 43) return tiff_fail(t, MQP_ERR_UNSUPPORTED, "BigTIFF files are not supported");
  if (magic != 42) return tiff_fail(t, MQP_ERR_INVALID, "not a TIFF file (magic number)");
  uint64_t ifd = rd32(t, 4);
  std::string err;
  while (ifd != 0) {
    if (ifd + 2 > t->size) return tiff_fail(t, MQP_ERR_INVALID, "IFD offset outside the file");
    if (t->pages.size() > (1u << 24)) return tiff_fail(t, MQP_ERR_INVALID, "too many pages (IFD loop?)");
    const uint16_t n = rd16(t, ifd);
    if (ifd + 2 + 12ull * n + 4 > t->size) return tiff_fail(t, MQP_ERR_INVALID, "IFD outside the file");
    Page pg;
    int spp = 1, planar = 1, predictor = 1;
    std::vector<uint64_t> v;
    for (int i = 0; i < n; ++i) {
      const size_t e = ifd + 2 + 12 * (size_t)i;
      const uint16_t tag = rd16(t, e);
      switch (tag) {
        case 256: case 257: case 258: case 259: case 273: case 277: case 278: case 279: case 284: case 317:
        case 322: case 323: case 324: case 325: case 339:
          if (!entry_values(t, e, v, err)) return tiff_fail(t, MQP_ERR_INVALID, err);
          break;
        default:
          continue;
      }
      if (v.empty()) return tiff_fail(t, MQP_ERR_INVALID, "empty TIFF field " + std::to_string(tag));
      switch (tag) {
        case 256: pg.width = (int64_t)v[0]; break;
        case 257: pg.height = (int64_t)v[0]; break;
        case 258: pg.bits = (int)v[0]; break;
        case 259: pg.compression = (int)v[0]; break;
        case 273: case 324: pg.offsets = v; break;
        case 277: spp = (int)v[0]; break;
        case 278: pg.rows_per_strip = (int64_t)v[0]; break;
        case 279: case 325: pg.counts = v; break;
        case 284: planar = (int)v[0]; break;
        case 317: predictor = (int)v[0]; break;
        case 322: pg.tile_w = (int64_t)v[0]; pg.tiled = true; break;
        case 323: pg.tile_h = (int64_t)v[0]; pg.tiled = true; break;
        case 339: pg.format = (int)v[0]; break;
      }
    }
    const std::string who = "page " + std::to_string(t->pages.size()) + ": ";
    if (pg.width < 1 || pg.height < 1) return tiff_fail(t, MQP_ERR_INVALID, who + "missing image size");
    if (spp != 1 || planar != 1)
      return tiff_fail(t, MQP_ERR_UNSUPPORTED, who + "only one sample per pixel is supported");
    if (predictor != 1) return tiff_fail(t, MQP_ERR_UNSUPPORTED, who + "differencing predictors are not supported");
    if (pg.compression != 1 && pg.compression != 32773)
      return tiff_fail(t, MQP_ERR_UNSUPPORTED,
                       who + "compression " + std::to_string(pg.compression) + " (only none and PackBits)");
    const bool ok_bits = (pg.format == 3) ? (pg.bits == 32 || pg.bits == 64)
                                          : ((pg.format == 1 || pg.format == 2) && (pg.bits == 8 || pg.bits == 16 || pg.bits == 32));
    if (!ok_bits) return tiff_fail(t, MQP_ERR_UNSUPPORTED, who + "unsupported sample format / bits");
    if (pg.tiled && (pg.tile_w < 1 || pg.tile_h < 1)) return tiff_fail(t, MQP_ERR_INVALID, who + "bad tile size");
    if (!pg.tiled && (pg.rows_per_strip < 1 || pg.rows_per_strip > pg.height)) pg.rows_per_strip = pg.height;
    const int64_t pieces = pg.tiled ? ((pg.width + pg.tile_w - 1) / pg.tile_w) * ((pg.height + pg.tile_h - 1) / pg.tile_h)
                                    : (pg.height + pg.rows_per_strip - 1) / pg.rows_per_strip;
    if ((int64_t)pg.offsets.size() != pieces || (int64_t)pg.counts.size() != pieces)
      return tiff_fail(t, MQP_ERR_INVALID, who + "strip/tile offsets and counts do not match the image");
    for (int64_t k = 0; k < pieces; ++k)
      if (pg.offsets[k] + pg.counts[k] > t->size) return tiff_fail(t, MQP_ERR_INVALID, who + "data outside the file");
    t->pages.push_back(std::move(pg));
    ifd = rd32(t, ifd + 2 + 12ull * n);
  }
  if (t->pages.empty()) return tiff_fail(t, MQP_ERR_INVALID, "TIFF file without pages");
  return MQP_OK;
}

// PackBits: n in [0, 127] copies n + 1 bytes, n in [-127, -1] repeats the
// next byte 1 - n times, -128 is skipped.
bool unpackbits(const uint8_t* src, size_t n, std::vector<uint8_t>& out, size_t want) {
  out.clear();
  out.reserve(want);
  size_t i = 0;
  while (i < n && out.size() < want) {
    const int8_t c = (int8_t)src[i++];
    if (c >= 0) {
      const size_t len = (size_t)c + 1;
      if (i + len > n) return false;
      out.insert(out.end(), src + i, src + i + len);
      i += len;
    } else if (c != -128) {
      if (i >= n) return false;
      out.insert(out.end(), (size_t)(1 - c), src[i++]);
    }
  }
  return out.size() >= want;
}

template <typename U>
U byteswap(U v) {
  U r;
  const uint8_t* a = (const uint8_t*)&v;
  uint8_t* b = (uint8_t*)&r;
  for (size_t i = 0; i < sizeof(U); ++i) b[i] = a[sizeof(U) - 1 - i];
  return r;
}

// One strip or tile (row-major, `rows` x `pw` samples of type S from src)
// into the column-major page at (r0, c0), clipped to H x W.
template <typename S, typename D>
void piece_to_page(const uint8_t* src, bool swap, int64_t rows, int64_t pw, int64_t r0, int64_t c0, int64_t H,
                   int64_t W, D* dst) {
  const int64_t yn = std::min(rows, H - r0), xn = std::min(pw, W - c0);
  for (int64_t x = 0; x < xn; ++x) {
    D* col = dst + (r0 + H * (c0 + x));
    for (int64_t y = 0; y < yn; ++y) {
      S v;
      memcpy(&v, src + (size_t)(y * pw + x) * sizeof(S), sizeof(S));
      if (swap) v = byteswap(v);
      col[y] = (D)v;
    }
  }
}

template <typename D>
void piece_dispatch(const Page& pg, const uint8_t* src, bool swap, int64_t rows, int64_t pw, int64_t r0, int64_t c0,
                    D* dst) {
  const int64_t H = pg.height, W = pg.width;
  if (pg.format == 3) {
    if (pg.bits == 32) piece_to_page<float, D>(src, swap, rows, pw, r0, c0, H, W, dst);
    else piece_to_page<double, D>(src, swap, rows, pw, r0, c0, H, W, dst);
  } else if (pg.format == 2) {
    if (pg.bits == 8) piece_to_page<int8_t, D>(src, swap, rows, pw, r0, c0, H, W, dst);
    else if (pg.bits == 16) piece_to_page<int16_t, D>(src, swap, rows, pw, r0, c0, H, W, dst);
    else piece_to_page<int32_t, D>(src, swap, rows, pw, r0, c0, H, W, dst);
  } else {
    if (pg.bits == 8) piece_to_page<uint8_t, D>(src, swap, rows, pw, r0, c0, H, W, dst);
    else if (pg.bits == 16) piece_to_page<uint16_t, D>(src, swap, rows, pw, r0, c0, H, W, dst);
    else piece_to_page<uint32_t, D>(src, swap, rows, pw, r0, c0, H, W, dst);
  }
}

// Page `k` into dst (column-major H x W of dtype), one strip or tile at a time.
int read_page(mqp_tiff* t, int64_t k, int dtype, void* dst, std::string& err) {
  const Page& pg = t->pages[k];
  const int bps = pg.bits / 8;
  const int64_t H = pg.height, W = pg.width;
  const int64_t pw = pg.tiled ? pg.tile_w : W;  // piece width in pixels
  const int64_t ph = pg.tiled ? pg.tile_h : pg.rows_per_strip;
  const int64_t across = pg.tiled ? (W + pw - 1) / pw : 1;
  std::vector<uint8_t> buf;
  for (size_t s = 0; s < pg.offsets.size(); ++s) {
    const int64_t r0 = (int64_t)(s / across) * ph, c0 = (int64_t)(s % across) * pw;
    const int64_t rows = pg.tiled ? ph : std::min(ph, H - r0);
    const size_t want = (size_t)(rows * pw * bps);
    const uint8_t* src = t->map + pg.offsets[s];
    if (pg.compression == 32773) {
      if (!unpackbits(src, pg.counts[s], buf, want)) {
        err = "page " + std::to_string(k) + ": corrupt PackBits data";
        return MQP_ERR_INVALID;
      }
      src = buf.data();
    } else if (pg.counts[s] < want) {
      err = "page " + std::to_string(k) + ": strip or tile shorter than its rows";
      return MQP_ERR_INVALID;
    }
    // row-major piece -> column-major page (byte-swapped for big-endian files)
    if (dtype == MQP_F32) piece_dispatch<float>(pg, src, t->big_endian, rows, pw, r0, c0, (float*)dst);
    else piece_dispatch<double>(pg, src, t->big_endian, rows, pw, r0, c0, (double*)dst);
  }
  return MQP_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// frame source: a reader thread filling a ring of pinned buffers
// ---------------------------------------------------------------------------
struct mqp_frame_source {
  mqp_tiff* tiff = nullptr;
  int64_t pages_per_frame = 1, frames = 0;
  int dtype = MQP_F32;
  size_t frame_bytes = 0;
  std::vector<void*> ring;
  bool pinned = false;
  std::thread reader;
  std::mutex mu;
  std::condition_variable cv;
  int64_t filled = 0;    // frames the reader has completed
  int64_t consumed = 0;  // frames handed out (the last one is still in use)
  bool stop = false;
  int error = MQP_OK;
  std::string last_error;
};

namespace {

void reader_loop(mqp_frame_source* s) {
  const size_t page_elems = (size_t)(s->tiff->pages[0].width * s->tiff->pages[0].height);
  const size_t es = s->dtype == MQP_F32 ? 4 : 8;
  for (int64_t f = 0; f < s->frames; ++f) {
    {
      // a buffer is free once the consumer has moved past the frame it held
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv.wait(lk, [&] { return s->stop || f - s->consumed < (int64_t)s->ring.size() - 1; });
      if (s->stop) return;
    }
    char* dst = (char*)s->ring[f % s->ring.size()];
    std::string err;
    int rc = MQP_OK;
    for (int64_t p = 0; p < s->pages_per_frame && rc == MQP_OK; ++p)
      rc = read_page(s->tiff, f * s->pages_per_frame + p, s->dtype, dst + p * page_elems * es, err);
    std::lock_guard<std::mutex> lk(s->mu);
    if (rc != MQP_OK) {
      s->error = rc;
      s->last_error = err;
      s->cv.notify_all();
      return;
    }
    s->filled = f + 1;
    s->cv.notify_all();
  }
}

}  // namespace

extern "C" {

int mqp_tiff_open(const char* path, mqp_tiff** out) {
  if (!path || !out) return MQP_ERR_INVALID;
  *out = nullptr;
  mqp_tiff* t = new mqp_tiff();
  t->fd = open(path, O_RDONLY);
  struct stat st;
  if (t->fd < 0 || fstat(t->fd, &st) != 0) {
    t->last_error = std::string("cannot open ") + path;
    *out = t;
    return MQP_ERR_NOT_FOUND;
  }
  t->size = (size_t)st.st_size;
  if (t->size > 0) {
    void* m = mmap(nullptr, t->size, PROT_READ, MAP_PRIVATE, t->fd, 0);
    if (m == MAP_FAILED) {
      t->last_error = std::string("cannot map ") + path;
      *out = t;
      return MQP_ERR_INVALID;
    }
    t->map = (const uint8_t*)m;
  }
  *out = t;
  return parse(t);
}

int mqp_tiff_get_info(const mqp_tiff* t, mqp_tiff_info* info) {
  if (!t || !info || t->pages.empty()) return MQP_ERR_INVALID;
  const Page& p = t->pages[0];
  info->width = p.width;
  info->height = p.height;
  info->pages = (int64_t)t->pages.size();
  info->bits = p.bits;
  info->sample_format = p.format;
  info->compression = p.compression;
  info->tiled = p.tiled ? 1 : 0;
  info->uniform = 1;
  for (const Page& q : t->pages)
    if (q.width != p.width || q.height != p.height) info->uniform = 0;
  return MQP_OK;
}

int mqp_tiff_read(mqp_tiff* t, int64_t first_page, int64_t npages, int dtype, void* dst) {
  if (!t || !dst) return tiff_fail(t, MQP_ERR_INVALID, "null argument");
  if (dtype != MQP_F32 && dtype != MQP_F64) return tiff_fail(t, MQP_ERR_INVALID, "dtype must be MQP_F32 or MQP_F64");
  if (first_page < 0 || npages < 0 || first_page + npages > (int64_t)t->pages.size())
    return tiff_fail(t, MQP_ERR_INVALID, "pages outside the file");
  if (npages == 0) return MQP_OK;
  const Page& p0 = t->pages[first_page];
  const size_t page_b = (size_t)(p0.width * p0.height) * (dtype == MQP_F32 ? 4 : 8);
  for (int64_t k = first_page; k < first_page + npages; ++k)
    if (t->pages[k].width != p0.width || t->pages[k].height != p0.height)
      return tiff_fail(t, MQP_ERR_INVALID, "pages of one read must share their size");
  // pages decode independently: spread them over a few threads
  const int nth = (int)std::min<int64_t>(npages, std::max(1u, std::min(8u, std::thread::hardware_concurrency())));
  std::vector<int> rcs(nth, MQP_OK);
  std::vector<std::string> errs(nth);
  auto work = [&](int w) {
    for (int64_t k = w; k < npages && rcs[w] == MQP_OK; k += nth)
      rcs[w] = read_page(t, first_page + k, dtype, (char*)dst + k * page_b, errs[w]);
  };
  std::vector<std::thread> th;
  for (int w = 1; w < nth; ++w) th.emplace_back(work, w);
  work(0);
  for (auto& x : th) x.join();
  for (int w = 0; w < nth; ++w)
    if (rcs[w] != MQP_OK) return tiff_fail(t, rcs[w], errs[w]);
  return MQP_OK;
}

const char* mqp_tiff_last_error(const mqp_tiff* t) { return t ? t->last_error.c_str() : "null TIFF handle"; }

int mqp_tiff_close(mqp_tiff* t) {
  if (!t) return MQP_OK;
  if (t->map) munmap((void*)t->map, t->size);
  if (t->fd >= 0) close(t->fd);
  delete t;
  return MQP_OK;
}

int mqp_frame_source_create(const char* path, int64_t pages_per_frame, int dtype, int ring, mqp_frame_source** out) {
  if (!out) return MQP_ERR_INVALID;
  *out = nullptr;
  if (pages_per_frame < 1 || ring < 2 || ring > 64 || (dtype != MQP_F32 && dtype != MQP_F64)) return MQP_ERR_INVALID;
  mqp_frame_source* s = new mqp_frame_source();
  *out = s;
  int rc = mqp_tiff_open(path, &s->tiff);
  if (rc != MQP_OK) {
    s->error = rc;
    s->last_error = s->tiff ? s->tiff->last_error : "cannot open the file";
    return rc;
  }
  mqp_tiff_info info;
  mqp_tiff_get_info(s->tiff, &info);
  if (!info.uniform) {
    s->last_error = "pages differ in size";
    return s->error = MQP_ERR_INVALID;
  }
  s->pages_per_frame = pages_per_frame;
  s->frames = info.pages / pages_per_frame;
  s->dtype = dtype;
  s->frame_bytes = (size_t)(info.width * info.height * pages_per_frame) * (dtype == MQP_F32 ? 4 : 8);
  // pinned buffers when a CUDA device is there (their copies to the device
  // run at full speed), pageable ones otherwise
  s->pinned = true;
  for (int i = 0; i < ring; ++i) {
    void* b = nullptr;
    if (s->pinned && cudaHostAlloc(&b, s->frame_bytes, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      s->pinned = false;
      for (void* q : s->ring) cudaFreeHost(q);
      s->ring.clear();
      i = -1;
      continue;
    }
    if (!s->pinned) b = aligned_alloc(4096, (s->frame_bytes + 4095) / 4096 * 4096);
    if (!b) {
      s->last_error = "cannot allocate the frame ring";
      return s->error = MQP_ERR_OOM;
    }
    s->ring.push_back(b);
  }
  s->reader = std::thread(reader_loop, s);
  return MQP_OK;
}

int mqp_frame_source_info(const mqp_frame_source* s, int64_t* frames, int64_t dims[3], int32_t* pinned) {
  if (!s || !s->tiff) return MQP_ERR_INVALID;
  if (frames) *frames = s->frames;
  if (dims) {
    dims[0] = s->tiff->pages[0].height;
    dims[1] = s->tiff->pages[0].width;
    dims[2] = s->pages_per_frame;
  }
  if (pinned) *pinned = s->pinned ? 1 : 0;
  return MQP_OK;
}

int mqp_frame_source_next(mqp_frame_source* s, const void** frame, int64_t* index) {
  if (!s || !frame) return MQP_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  if (s->error != MQP_OK && s->filled <= s->consumed) return s->error;
  if (s->consumed >= s->frames) return MQP_ERR_NOT_FOUND;
  s->cv.wait(lk, [&] { return s->filled > s->consumed || s->error != MQP_OK; });
  if (s->filled <= s->consumed) return s->error;
  const int64_t f = s->consumed++;
  s->cv.notify_all();
  *frame = s->ring[f % s->ring.size()];
  if (index) *index = f;
  return MQP_OK;
}

const char* mqp_frame_source_last_error(const mqp_frame_source* s) {
  return s ? s->last_error.c_str() : "null frame source";
}

int mqp_frame_source_destroy(mqp_frame_source* s) {
  if (!s) return MQP_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv.notify_all();
  }
  if (s->reader.joinable()) s->reader.join();
  for (void* b : s->ring) {
    if (s->pinned) cudaFreeHost(b);
    else free(b);
  }
  mqp_tiff_close(s->tiff);
  delete s;
  return MQP_OK;
}

}  // extern "C"
