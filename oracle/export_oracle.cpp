// CPU oracle for the pipeline's file ends: the SLC measurement TIFF reader,
// dB conversion, dB statistics, overview downsampling and the
// Cloud-Optimised GeoTIFF writer.
//
// TEST INFRASTRUCTURE ONLY (the parity tests' reference results and the CPU baseline): a plain
// sequential restatement of the reference's arithmetic and file layout,
// never linked into the product library.
//
//   to_db_inplace          sardine/src/export.rs:59-99
//   compute_db_stats       sardine/src/run.rs:63-97
//   downsample_2x          sardine/src/export.rs:362-392
//   write_cog_with_crs     sardine/src/export.rs:329-355
//   write_cog_raw_inner    sardine/src/export.rs:417-760
//   geo_key_directory      sardine/src/output_crs.rs:265-287
//   SlcReader              sardine/src/slc_reader.rs:268-583
//   apply_multilook        sardine/src/scene_prep.rs:1060-1160
//   to_ground_range        sardine/src/ground_range.rs:148-485
//   deramp_subswath        sardine/src/insar/deramp.rs:114-276
//   resample_secondary     sardine/src/insar/coreg.rs:230-264, 428-466
//   ecef_from_slant_range_doppler  sardine/src/insar/coreg.rs:280-362
//   form_interferogram     sardine/src/insar/interferogram.rs:165-398
//   compute_coreg_offsets  sardine/src/insar/coreg.rs:128-223, 371-414, 478-568
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../include/sardine_b200.h"

namespace {

// GeoKeyDirectoryTag payload (output_crs.rs:265-287).
std::vector<uint16_t> geo_keys(int crs, int zone) {
  if (crs == SD_CRS_WGS84) return {1, 1, 0, 3, 1024, 0, 1, 2, 1025, 0, 1, 1, 2048, 0, 1, 4326};
  const uint16_t epsg = (uint16_t)((crs == SD_CRS_UTM_SOUTH ? 32700 : 32600) + zone);
  return {1, 1, 0, 4, 1024, 0, 1, 1, 1025, 0, 1, 1, 3072, 0, 1, epsg, 3076, 0, 1, 9001};
}

// export.rs:362-392: each destination pixel is the f64 mean of the non-NaN,
// in-range pixels of its 2x2 source patch (row-major order), NaN when none.
std::vector<float> downsample(const std::vector<float> &src, uint64_t c, uint64_t r, uint64_t *dc,
                              uint64_t *dr) {
  const uint64_t oc = (c + 1) / 2, orows = (r + 1) / 2;
  std::vector<float> dst(oc * orows, NAN);
  for (uint64_t y = 0; y < orows; ++y)
    for (uint64_t x = 0; x < oc; ++x) {
      double sum = 0.0;
      uint32_t cnt = 0;
      for (uint64_t a = 0; a < 2; ++a)
        for (uint64_t b = 0; b < 2; ++b) {
          const uint64_t sy = 2 * y + a, sx = 2 * x + b;
          if (sy < r && sx < c) {
            const float v = src[sy * c + sx];
            if (!std::isnan(v)) {
              sum += (double)v;
              cnt += 1;
            }
          }
        }
      if (cnt > 0) dst[y * oc + x] = (float)(sum / (double)cnt);
    }
  *dc = oc;
  *dr = orows;
  return dst;
}

struct Out {
  FILE *f;
  bool ok = true;
  void bytes(const void *p, size_t n) {
    if (ok && fwrite(p, 1, n, f) != n) ok = false;
  }
  void u16(uint16_t v) { bytes(&v, 2); }
  void u32(uint32_t v) { bytes(&v, 4); }
  void u64(uint64_t v) { bytes(&v, 8); }
  void f64(double v) { bytes(&v, 8); }
};

}  // namespace

extern "C" {

// to_db_inplace: NaN kept; v <= floor -> NaN (noise-masked); else 10 log10 v.
int orc_to_db_inplace(float *data, uint64_t n, float noise_floor_linear, uint64_t *converted,
                      uint64_t *masked) {
  if (noise_floor_linear < 0.0f) return SD_ERR_EXPORT_INVALID_NOISE_FLOOR;
  uint64_t cv = 0, nm = 0;
  for (uint64_t i = 0; i < n; ++i) {
    const float v = data[i];
    if (std::isnan(v)) continue;
    if (v <= noise_floor_linear) {
      data[i] = NAN;
      ++nm;
    } else {
      data[i] = 10.0f * std::log10(v);
      ++cv;
    }
  }
  *converted = cv;
  *masked = nm;
  return SD_OK;
}

// compute_db_stats: min, max, f64 mean of the finite values, and the median
// of every stride-th finite value (stride = max(n_finite / 100000, 1)).
void orc_db_stats(const float *data, uint64_t n, float *out) {
  float mn = INFINITY, mx = -INFINITY;
  double sum = 0.0;
  uint64_t cnt = 0;
  for (uint64_t i = 0; i < n; ++i) {
    const float v = data[i];
    if (!std::isfinite(v)) continue;
    if (v < mn) mn = v;
    if (v > mx) mx = v;
    sum += (double)v;
    ++cnt;
  }
  if (cnt == 0) {
    out[0] = out[1] = out[2] = out[3] = NAN;
    return;
  }
  const uint64_t stride = std::max<uint64_t>(cnt / 100000, 1);
  std::vector<float> sample;
  uint64_t k = 0;
  for (uint64_t i = 0; i < n; ++i) {
    const float v = data[i];
    if (!std::isfinite(v)) continue;
    if (k % stride == 0) sample.push_back(v);
    ++k;
  }
  std::sort(sample.begin(), sample.end());
  out[0] = mn;
  out[1] = mx;
  out[2] = (float)(sum / (double)cnt);
  out[3] = sample[sample.size() / 2];
}

void orc_downsample_2x(const float *src, uint64_t cols, uint64_t rows, float *dst) {
  std::vector<float> s(src, src + cols * rows);
  uint64_t dc, dr;
  std::vector<float> d = downsample(s, cols, rows, &dc, &dr);
  std::memcpy(dst, d.data(), d.size() * sizeof(float));
}

// write_cog_with_crs / write_cog_raw_inner.
int orc_write_cog(const char *path, const float *data, uint64_t cols, uint64_t rows, const double *gt,
                  int crs, int zone, uint32_t tile_size) {
  const double pw = gt[1], ph = -gt[5];
  if (!std::isfinite(pw) || pw <= 0.0 || !std::isfinite(ph) || ph <= 0.0) return SD_ERR_EXPORT_INVALID_GEOTRANSFORM;
  if (tile_size < 64 || tile_size > 4096 || (tile_size & (tile_size - 1)) != 0) return SD_ERR_EXPORT_INVALID_TILE_SIZE;
  const std::vector<uint16_t> keys = geo_keys(crs, zone);
  const uint64_t ts = tile_size;

  // overview pyramid: finest first, then reversed (coarsest first)
  struct Level {
    std::vector<float> d;
    uint64_t c, r;
  };
  std::vector<Level> ov;
  {
    std::vector<float> full(data, data + cols * rows);
    uint64_t c, r;
    std::vector<float> cur = downsample(full, cols, rows, &c, &r);
    while (c > ts || r > ts) {
      ov.push_back({cur, c, r});
      uint64_t c2, r2;
      std::vector<float> nxt = downsample(cur, c, r, &c2, &r2);
      cur = std::move(nxt);
      c = c2;
      r = r2;
    }
    ov.push_back({cur, c, r});
  }
  std::reverse(ov.begin(), ov.end());

  const bool big = rows * cols * 4ull > 0xFFFFFFFFull;
  auto grid = [&](uint64_t c, uint64_t r) { return ((c + ts - 1) / ts) * ((r + ts - 1) / ts); };
  const uint64_t entries = 17;
  const uint64_t ifd_bytes = big ? 8 + entries * 20 + 8 : 2 + entries * 12 + 4;
  const uint64_t arr_entry = big ? 8 : 4;
  uint64_t off = big ? 16 : 8;

  std::vector<std::pair<uint64_t, uint64_t>> dims;
  for (const Level &l : ov) dims.push_back({l.c, l.r});
  dims.push_back({cols, rows});
  std::vector<uint64_t> ifd_off, toff_off, tbc_off, ntiles;
  for (auto &cr : dims) {
    ifd_off.push_back(off);
    off += ifd_bytes;
    const uint64_t nt = grid(cr.first, cr.second);
    toff_off.push_back(off);
    off += nt * arr_entry;
    tbc_off.push_back(off);
    off += nt * arr_entry;
    ntiles.push_back(nt);
  }
  const uint64_t scale_off = off;
  off += 24;
  const uint64_t tie_off = off;
  off += 48;
  const uint64_t keys_off = off;
  off += keys.size() * 2;
  const uint64_t tile_bytes = ts * ts * 4;
  std::vector<uint64_t> data_start;
  for (uint64_t nt : ntiles) {
    data_start.push_back(off);
    off += nt * tile_bytes;
  }

  Out o{std::fopen(path, "wb")};
  if (!o.f) return SD_ERR_EXPORT_IO;
  o.bytes("II", 2);
  if (big) {
    o.u16(43);
    o.u16(8);
    o.u16(0);
    o.u64(ifd_off[0]);
  } else {
    o.u16(42);
    o.u32((uint32_t)ifd_off[0]);
  }
  const size_t n_ifd = dims.size();
  for (size_t k = 0; k < n_ifd; ++k) {
    const uint64_t c = dims[k].first, r = dims[k].second, nt = ntiles[k];
    const uint64_t next = k + 1 < n_ifd ? ifd_off[k + 1] : 0;
    auto e = [&](uint16_t tag, uint16_t typ, uint64_t count, uint64_t val) {
      o.u16(tag);
      o.u16(typ);
      if (big) {
        o.u64(count);
        o.u64(val);
      } else {
        o.u32((uint32_t)count);
        o.u32((uint32_t)val);
      }
    };
    if (big) o.u64(entries);
    else o.u16((uint16_t)entries);
    e(256, 4, 1, c);
    e(257, 4, 1, r);
    e(258, 3, 1, 32);
    e(259, 3, 1, 1);
    e(262, 3, 1, 1);
    e(277, 3, 1, 1);
    if (big) {
      e(282, 5, 1, (1ull << 32) | 72ull);
      e(283, 5, 1, (1ull << 32) | 72ull);
    } else {
      e(282, 4, 1, 72);
      e(283, 4, 1, 72);
    }
    e(296, 3, 1, 1);
    e(322, 4, 1, ts);
    e(323, 4, 1, ts);
    e(324, big ? 16 : 4, nt, toff_off[k]);
    e(325, big ? 16 : 4, nt, tbc_off[k]);
    e(339, 3, 1, 3);
    e(33550, 12, 3, scale_off);
    e(33922, 12, 6, tie_off);
    e(34735, 3, keys.size(), keys_off);
    if (big) o.u64(next);
    else o.u32((uint32_t)next);
    for (uint64_t t = 0; t < nt; ++t) {
      if (big) o.u64(data_start[k] + t * tile_bytes);
      else o.u32((uint32_t)(data_start[k] + t * tile_bytes));
    }
    for (uint64_t t = 0; t < nt; ++t) {
      if (big) o.u64(tile_bytes);
      else o.u32((uint32_t)tile_bytes);
    }
  }
  o.f64(gt[1]);
  o.f64(-gt[5]);
  o.f64(0.0);
  o.f64(0.0);
  o.f64(0.0);
  o.f64(0.0);
  o.f64(gt[0]);
  o.f64(gt[3]);
  o.f64(0.0);
  for (uint16_t k : keys) o.u16(k);

  std::vector<float> tile(ts * ts);
  for (size_t k = 0; k < n_ifd; ++k) {
    const float *src = k + 1 < n_ifd ? ov[k].d.data() : data;
    const uint64_t c = dims[k].first, r = dims[k].second;
    const uint64_t nx = (c + ts - 1) / ts, ny = (r + ts - 1) / ts;
    for (uint64_t ty = 0; ty < ny; ++ty)
      for (uint64_t tx = 0; tx < nx; ++tx) {
        std::fill(tile.begin(), tile.end(), NAN);
        const uint64_t r0 = ty * ts, c0 = tx * ts;
        const uint64_t r1 = std::min(r0 + ts, r), c1 = std::min(c0 + ts, c);
        for (uint64_t y = r0; y < r1; ++y)
          std::memcpy(&tile[(y - r0) * ts], src + y * c + c0, (c1 - c0) * sizeof(float));
        o.bytes(tile.data(), tile_bytes);
      }
  }
  const bool ok = o.ok;
  if (std::fclose(o.f) != 0 || !ok) return SD_ERR_EXPORT_IO;
  return SD_OK;
}

}  // extern "C"

// ── SLC measurement TIFF reader (slc_reader.rs:268-583) ─────────────────────
// parse_ifd's checks in its order, then read_burst_raw of [first, first+n)
// rows into out (n * width * 2 int16, host byte order).  width/height are
// filled once the IFD is accepted; out may be null to only open the file.
namespace {
uint16_t o_rd16(const unsigned char *b, bool le) {
  return le ? (uint16_t)(b[0] | (b[1] << 8)) : (uint16_t)(b[1] | (b[0] << 8));
}
uint32_t o_rd32(const unsigned char *b, bool le) {
  uint32_t v = 0;
  for (int k = 0; k < 4; ++k) v |= (uint32_t)b[le ? k : 3 - k] << (8 * k);
  return v;
}
bool o_read(FILE *f, uint64_t off, void *dst, size_t n) {
  return std::fseek(f, (long)off, SEEK_SET) == 0 && std::fread(dst, 1, n, f) == n;
}
}  // namespace

extern "C" int orc_slc_read(const char *path, uint64_t first, uint64_t n, int16_t *out, uint32_t *width_out,
                            uint32_t *height_out) {
  FILE *f = std::fopen(path, "rb");
  if (!f) return SD_ERR_SLC_IO;
  struct C {
    FILE *f;
    ~C() { std::fclose(f); }
  } closer{f};
  unsigned char h[8];
  if (!o_read(f, 0, h, 8)) return SD_ERR_SLC_IO;
  bool le;
  if (h[0] == 'I' && h[1] == 'I') le = true;
  else if (h[0] == 'M' && h[1] == 'M') le = false;
  else return SD_ERR_SLC_NOT_TIFF;
  const uint16_t magic = o_rd16(h + 2, le);
  if (magic == 43) return SD_ERR_SLC_BIGTIFF;
  if (magic != 42) return SD_ERR_SLC_NOT_TIFF;
  const uint64_t ifd = o_rd32(h + 4, le);
  unsigned char nb[2];
  if (!o_read(f, ifd, nb, 2)) return SD_ERR_SLC_IO;
  const size_t ne = o_rd16(nb, le);
  std::vector<unsigned char> e(ne * 12);
  if (ne && !o_read(f, ifd + 2, e.data(), e.size())) return SD_ERR_SLC_IO;
  long width = -1, height = -1, bps = -1, comp = -1, rps = -1, spp = -1, sfmt = -1;
  bool so = false;
  uint16_t so_type = 0;
  uint32_t so_count = 0, so_val = 0;
  for (size_t k = 0; k < ne; ++k) {
    const unsigned char *p = &e[12 * k];
    const uint16_t tag = o_rd16(p, le), typ = o_rd16(p + 2, le);
    const uint32_t cnt = o_rd32(p + 4, le);
    long v = typ == 3 ? (long)o_rd16(p + 8, le) : (typ == 4 ? (long)o_rd32(p + 8, le) : -1);
    switch (tag) {
      case 256: width = v; break;
      case 257: height = v; break;
      case 258: bps = v; break;
      case 259: comp = v; break;
      case 278: rps = v; break;
      case 277: spp = v; break;
      case 339: sfmt = v; break;
      case 273:
        so = true;
        so_type = typ;
        so_count = cnt;
        so_val = o_rd32(p + 8, le);
        break;
      default: break;
    }
  }
  if (width < 0 || height < 0 || bps < 0 || comp < 0 || rps < 0 || sfmt < 0 || !so) return SD_ERR_SLC_MISSING_TAG;
  if (spp < 0) spp = 1;
  if ((uint16_t)comp != 1 || (uint16_t)sfmt != 5 || (uint16_t)bps != 32 || rps != 1 || (uint16_t)spp != 1 ||
      so_count != (uint32_t)height || height == 0)
    return SD_ERR_SLC_UNSUPPORTED_FORMAT;
  const uint64_t row = (uint64_t)width * 4;
  uint64_t base = so_val, last = so_val;
  if (so_count > 1) {
    if (so_type != 3 && so_type != 4) return SD_ERR_SLC_UNSUPPORTED_FORMAT;
    const size_t each = so_type == 3 ? 2 : 4;
    unsigned char b[4];
    if (!o_read(f, so_val, b, each)) return SD_ERR_SLC_IO;
    base = each == 2 ? o_rd16(b, le) : o_rd32(b, le);
    if (!o_read(f, so_val + (uint64_t)(so_count - 1) * each, b, each)) return SD_ERR_SLC_IO;
    last = each == 2 ? o_rd16(b, le) : o_rd32(b, le);
  }
  if (last != base + (uint64_t)(height - 1) * row) return SD_ERR_SLC_NON_CONTIGUOUS_STRIPS;
  if (width_out) *width_out = (uint32_t)width;
  if (height_out) *height_out = (uint32_t)height;
  if (!out) return SD_OK;
  if (first > (uint64_t)height || n > (uint64_t)height - first) return SD_ERR_SLC_LINE_OUT_OF_BOUNDS;
  if (n == 0) return SD_OK;
  if (!o_read(f, base + first * row, out, n * row)) return SD_ERR_SLC_IO;
  if (!le)
    for (uint64_t i = 0; i < n * (uint64_t)width * 2; ++i) {
      const uint16_t u = (uint16_t)out[i];
      out[i] = (int16_t)(uint16_t)((u >> 8) | (u << 8));
    }
  return SD_OK;
}

// ── pre-TC multilook (scene_prep.rs:1060-1160, the boxcar part) ────────────
extern "C" int orc_multilook(const float *d, const float *nz, uint64_t lines, uint64_t samples, uint32_t rl,
                             uint32_t al, float *od, float *onz) {
  if (rl == 0 || al == 0) return SD_ERR_INVALID_ARGUMENT;
  const uint64_t ol = lines / al, os = samples / rl;
  if (ol == 0 || os == 0) return SD_ERR_INVALID_ARGUMENT;
  for (uint64_t y = 0; y < ol; ++y)
    for (uint64_t x = 0; x < os; ++x) {
      double s = 0.0, sn = 0.0;
      uint32_t c = 0;
      for (uint32_t a = 0; a < al; ++a)
        for (uint32_t r = 0; r < rl; ++r) {
          const uint64_t k = (y * al + a) * samples + x * rl + r;
          if (!std::isnan(d[k])) {
            s += (double)d[k];
            sn += (double)nz[k];
            ++c;
          }
        }
      od[y * os + x] = c ? (float)(s / (double)c) : NAN;
      onz[y * os + x] = c ? (float)(sn / (double)c) : NAN;
    }
  return SD_OK;
}

// ── ground range (ground_range.rs:148-485) ──────────────────────────────────
// The reference's structure: per-swath range interpolators at the
// mid-azimuth grid row, the per-column incidence profile, cumulative ground
// range, the column mapping, the full projected image, then the azimuth
// multilook.
namespace {
struct ORange {
  std::vector<double> t, a;
  double lo, hi;
  bool eval(double st, double *out) const {  // RangeInterpolator::interpolate
    if (st < lo || st > hi) return false;
    size_t b = 0, e = t.size();            // binary search: first index with t >= st
    while (b < e) {
      const size_t m = (b + e) / 2;
      if (t[m] < st) b = m + 1;
      else e = m;
    }
    if (b < t.size() && t[b] == st) {
      *out = a[b];
      return true;
    }
    if (b == 0) {
      *out = a[0];
      return true;
    }
    if (b >= t.size()) {
      *out = a[t.size() - 1];
      return true;
    }
    const double f = (st - t[b - 1]) / (t[b] - t[b - 1]);
    *out = a[b - 1] + f * (a[b] - a[b - 1]);
    return true;
  }
};
}  // namespace

extern "C" int orc_to_ground_range(const float *data, uint64_t lines, uint64_t samples, double near_t, double rps_s,
                                   double rps_m, const sd_grd_swath_grid *grids, int32_t n_grids, double target,
                                   double az_spacing, float *out, sd_grd_info *info) {
  if (lines == 0 || samples == 0) return SD_ERR_GRD_EMPTY_IMAGE;
  if (target <= 0.0) return SD_ERR_GRD_INVALID_SPACING;
  if (!std::isfinite(az_spacing) || az_spacing <= 0.0) return SD_ERR_GRD_INVALID_AZIMUTH_SPACING;
  std::vector<ORange> rs;
  for (int32_t g = 0; g < n_grids; ++g) {
    if (grids[g].n_points == 0) return SD_ERR_GRD_NO_GRID_POINTS;
    std::vector<uint32_t> ls;
    for (uint64_t k = 0; k < grids[g].n_points; ++k) ls.push_back(grids[g].points[k].line);
    std::sort(ls.begin(), ls.end());
    ls.erase(std::unique(ls.begin(), ls.end()), ls.end());
    const uint32_t mid = ls[ls.size() / 2];
    std::vector<std::pair<double, double>> v;
    for (uint64_t k = 0; k < grids[g].n_points; ++k)
      if (grids[g].points[k].line == mid)
        v.push_back({grids[g].points[k].slant_range_time_s, grids[g].points[k].incidence_angle_deg});
    std::stable_sort(v.begin(), v.end(), [](const std::pair<double, double> &x, const std::pair<double, double> &y) {
      return x.first < y.first;
    });
    ORange r;
    for (auto &q : v) {
      r.t.push_back(q.first);
      r.a.push_back(q.second);
    }
    r.lo = r.t.front();
    r.hi = r.t.back();
    rs.push_back(r);
  }
  std::stable_sort(rs.begin(), rs.end(), [](const ORange &x, const ORange &y) { return x.lo < y.lo; });
  std::vector<double> ang(samples);
  for (uint64_t c = 0; c < samples; ++c) {
    const double st = near_t + (double)c * rps_s;
    bool got = false;
    double best = 0.0, bd = 0.0;
    for (const ORange &r : rs) {
      double a;
      if (r.eval(st, &a)) {
        const double d = std::fabs(st - (r.lo + r.hi) / 2.0);
        if (!got || d < bd) {
          got = true;
          bd = d;
          best = a;
        }
      }
    }
    if (!got) {
      const ORange *nr = nullptr;
      double nd = 0.0;
      for (const ORange &r : rs) {
        const double d = st < r.lo ? r.lo - st : st - r.hi;
        if (!nr || d < nd) {
          nr = &r;
          nd = d;
        }
      }
      if (!nr || !(nd < (nr->hi - nr->lo) * 0.01) || !nr->eval(std::min(std::max(st, nr->lo), nr->hi), &best))
        return SD_ERR_GRD_INTERPOLATION_FAILED;
    }
    ang[c] = best * (M_PI / 180.0);
  }
  std::vector<double> gsp(samples), cum;
  for (uint64_t c = 0; c < samples; ++c) gsp[c] = rps_m / std::sin(ang[c]);
  double acc = 0.0;
  cum.push_back(0.0);
  for (uint64_t c = 1; c < samples; ++c) {
    acc += (gsp[c - 1] + gsp[c]) / 2.0;
    cum.push_back(acc);
  }
  const uint64_t os = (uint64_t)std::floor(cum.back() / target);
  if (os == 0) return SD_ERR_GRD_INVALID_SPACING;
  const uint64_t al = (uint64_t)std::max(std::round(target / az_spacing), 1.0);
  const uint64_t ol = lines / al;
  info->lines = ol;
  info->samples = os;
  info->range_pixel_spacing_m = target;
  info->azimuth_pixel_spacing_m = az_spacing * (double)al;
  info->range_looks = 1;
  info->azimuth_looks = al;
  if (!out) return SD_OK;
  // mapping: (left, right, frac); left == right means Exact
  std::vector<uint64_t> ml(os), mr(os);
  std::vector<double> mf(os, 0.0);
  uint64_t start = 0;
  for (uint64_t j = 0; j < os; ++j) {
    const double tg = (double)j * target;
    uint64_t b = start, e = samples;
    while (b < e) {
      const uint64_t m = (b + e) / 2;
      if (cum[m] < tg) b = m + 1;
      else e = m;
    }
    if (b < samples && cum[b] == tg) {
      ml[j] = mr[j] = b;
      start = b;
    } else if (b == 0) {
      ml[j] = mr[j] = 0;
    } else if (b >= samples) {
      ml[j] = mr[j] = samples - 1;
    } else {
      ml[j] = b - 1;
      mr[j] = b;
      mf[j] = (tg - cum[b - 1]) / (cum[b] - cum[b - 1]);
      start = b - 1;
    }
  }
  std::vector<float> proj(lines * os, NAN);
  for (uint64_t l = 0; l < lines; ++l)
    for (uint64_t j = 0; j < os; ++j) {
      const float *row = data + l * samples;
      float v;
      if (ml[j] == mr[j]) {
        v = row[ml[j]];
      } else {
        const float v0 = row[ml[j]], v1 = row[mr[j]];
        v = (std::isnan(v0) || std::isnan(v1)) ? NAN : v0 + (v1 - v0) * (float)mf[j];
      }
      proj[l * os + j] = v;
    }
  for (uint64_t o = 0; o < ol; ++o)
    for (uint64_t j = 0; j < os; ++j) {
      double s = 0.0;
      uint32_t c = 0;
      for (uint64_t l = o * al; l < o * al + al; ++l) {
        const float v = proj[l * os + j];
        if (!std::isnan(v)) {
          s += (double)v;
          ++c;
        }
      }
      out[o * os + j] = c ? (float)(s / (double)c) : NAN;
    }
  return SD_OK;
}

// deramp_subswath (insar/deramp.rs:114-210) with interp_dc_poly (227-276):
// the column times, the per-line interpolated polynomials, then one
// sequential pass over the pixels with the C library's sin and cos.
namespace {
int orc_interp_dc(const sd_dc_estimate *e, const std::vector<double> &et, double t, double q[4], double *bad_t) {
  const size_t n = et.size();
  const sd_dc_estimate *pick = nullptr;
  if (t < et[0]) {
    if (et[0] - t > 2.0) {
      *bad_t = t;
      return SD_ERR_INSAR_AZIMUTH_TIME_BEFORE_DC;
    }
    pick = &e[0];
  } else if (t >= et[n - 1]) {
    pick = &e[n - 1];
  }
  if (pick) {
    q[0] = pick->data_dc_poly[0];
    q[1] = pick->data_dc_poly[1];
    q[2] = pick->data_dc_poly[2];
    q[3] = pick->t0_s;
    return SD_OK;
  }
  size_t k = n - 2;
  for (size_t j = 0; j + 1 < n; ++j)
    if (t >= et[j] && t < et[j + 1]) {
      k = j;
      break;
    }
  const double a = (t - et[k]) / (et[k + 1] - et[k]);
  for (int j = 0; j < 3; ++j) q[j] = e[k].data_dc_poly[j] + (e[k + 1].data_dc_poly[j] - e[k].data_dc_poly[j]) * a;
  q[3] = e[k].t0_s + (e[k + 1].t0_s - e[k].t0_s) * a;
  return SD_OK;
}
}  // namespace

extern "C" int orc_deramp(const int16_t *iq, uint64_t lines, uint64_t samples, uint64_t col_off, double near_tau,
                          double rps_m, double ati, const sd_dc_estimate *est, uint64_t n_est, int64_t start_us,
                          float *out, double *bad_t) {
  if (n_est == 0) return SD_ERR_INSAR_NO_DC_ESTIMATES;
  const double dtau = 2.0 * rps_m / 299792458.0;
  std::vector<double> tau(samples);
  for (uint64_t c = 0; c < samples; ++c) tau[c] = near_tau + (double)(c + col_off) * dtau;
  std::vector<double> et(n_est);
  for (uint64_t k = 0; k < n_est; ++k) et[k] = (double)(est[k].azimuth_time_us - start_us) / 1e6;
  std::vector<double> poly(4 * lines);
  for (uint64_t l = 0; l < lines; ++l) {
    const int rc = orc_interp_dc(est, et, (double)l * ati, &poly[4 * l], bad_t);
    if (rc) return rc;
  }
  const double two_pi = 6.283185307179586;
  for (uint64_t l = 0; l < lines; ++l) {
    const double *q = &poly[4 * l];
    const double t_az = (double)l * ati;
    for (uint64_t c = 0; c < samples; ++c) {
      const double dt = tau[c] - q[3];
      const double f_dc = q[0] + q[1] * dt + q[2] * dt * dt;
      const double phi = two_pi * f_dc * t_az;
      const double sp = std::sin(phi), cp = std::cos(phi);
      const uint64_t i = l * samples + c;
      const double iv = iq[2 * i], qv = iq[2 * i + 1];
      out[2 * i] = (float)(iv * cp + qv * sp);
      out[2 * i + 1] = (float)(qv * cp - iv * sp);
    }
  }
  return SD_OK;
}

// ── InSAR: co-registration resampling and interferogram ──────────────────
extern "C" int orc_interpolate_orbit_and_accel(const sd_state_vector *svs, uint64_t n, int64_t t, double *pos,
                                               double *vel, double *acc);

namespace {
// eval_poly6 (coreg.rs:462-464)
double orc_poly6(const double *p, double l, double c) {
  return p[0] + p[1] * l + p[2] * c + p[3] * l * l + p[4] * l * c + p[5] * c * c;
}

// bilinear (coreg.rs:428-456); `l as usize` of NaN is 0 in Rust
void orc_bilinear(const float *sec, uint64_t lines, uint64_t samples, double l, double c, float *o) {
  o[0] = o[1] = 0.0f;
  if (l < 0.0 || c < 0.0) return;
  const double lf = std::floor(l), cf = std::floor(c);
  // `as usize`: NaN -> 0; indices at or past the end only need to fail the bounds test below
  const uint64_t l0 = lf == lf ? (lf < (double)lines ? (uint64_t)lf : lines) : 0;
  const uint64_t c0 = cf == cf ? (cf < (double)samples ? (uint64_t)cf : samples) : 0;
  const uint64_t l1 = l0 + 1, c1 = c0 + 1;
  if (l1 >= lines || c1 >= samples) return;
  const float wl = (float)(l - (double)l0), wc = (float)(c - (double)c0);
  auto lerp = [](float a, float b, float t) { return a + (b - a) * t; };
  for (int k = 0; k < 2; ++k) {
    const float p00 = sec[2 * (l0 * samples + c0) + k], p01 = sec[2 * (l0 * samples + c1) + k];
    const float p10 = sec[2 * (l1 * samples + c0) + k], p11 = sec[2 * (l1 * samples + c1) + k];
    o[k] = lerp(lerp(p00, p01, wc), lerp(p10, p11, wc), wl);
  }
}
}  // namespace

extern "C" int orc_resample_secondary(const float *sec, uint64_t sec_lines, uint64_t sec_samples, uint64_t lines,
                                      uint64_t samples, const double *az, const double *rg, float *out) {
  for (uint64_t l = 0; l < lines; ++l)
    for (uint64_t c = 0; c < samples; ++c) {
      const double lf = (double)l, cf = (double)c;
      const double ls = lf + orc_poly6(az, lf, cf), cs = cf + orc_poly6(rg, lf, cf);
      orc_bilinear(sec, sec_lines, sec_samples, ls, cs, out + 2 * (l * samples + c));
    }
  return SD_OK;
}

// ecef_from_slant_range_doppler (coreg.rs:280-362): 0 and the point, or 1.
extern "C" int orc_ecef_from_slant_range_doppler(const double *sat_pos, const double *sat_vel, double range_m,
                                                 uint64_t max_iter, double tol_m, double *out) {
  const double px = sat_pos[0], py = sat_pos[1], pz = sat_pos[2];
  const double vx = sat_vel[0], vy = sat_vel[1], vz = sat_vel[2];
  const double r = range_m, a = 6378137.0, b = 6356752.314245;
  const double sat_r = std::sqrt(px * px + py * py + pz * pz);
  const double scale = a / sat_r;
  double tx = px * scale, ty = py * scale, tz = pz * scale * (b / a);
  for (uint64_t it = 0; it < max_iter; ++it) {
    const double dx = tx - px, dy = ty - py, dz = tz - pz;
    const double f1 = dx * vx + dy * vy + dz * vz;
    const double f2 = dx * dx + dy * dy + dz * dz - r * r;
    const double f3 = tx * tx / (a * a) + ty * ty / (a * a) + tz * tz / (b * b) - 1.0;
    const double j00 = vx, j01 = vy, j02 = vz;
    const double j10 = 2.0 * dx, j11 = 2.0 * dy, j12 = 2.0 * dz;
    const double j20 = 2.0 * tx / (a * a), j21 = 2.0 * ty / (a * a), j22 = 2.0 * tz / (b * b);
    const double det = j00 * (j11 * j22 - j12 * j21) - j01 * (j10 * j22 - j12 * j20) + j02 * (j10 * j21 - j11 * j20);
    if (std::fabs(det) < 1e-20) return 1;
    const double dxt = (f1 * (j11 * j22 - j12 * j21) - j01 * (f2 * j22 - j12 * f3) + j02 * (f2 * j21 - j11 * f3)) / det;
    const double dyt = (j00 * (f2 * j22 - j12 * f3) - f1 * (j10 * j22 - j12 * j20) + j02 * (j10 * f3 - f2 * j20)) / det;
    const double dzt = (j00 * (j11 * f3 - f2 * j21) - j01 * (j10 * f3 - f2 * j20) + f1 * (j10 * j21 - j11 * j20)) / det;
    tx -= dxt;
    ty -= dyt;
    tz -= dzt;
    if (std::sqrt(dxt * dxt + dyt * dyt + dzt * dzt) < tol_m) {
      out[0] = tx, out[1] = ty, out[2] = tz;
      return 0;
    }
  }
  return 1;
}

// form_interferogram (interferogram.rs:165-398), its three loops in turn.
extern "C" int orc_form_interferogram(const float *ref, const float *sec, uint64_t lines, uint64_t samples,
                                      uint64_t col_off, double srt, double rps_m, double ati,
                                      const sd_state_vector *ref_svs, uint64_t n_ref, int64_t first_us,
                                      const sd_state_vector *sec_svs, uint64_t n_sec, double wavelength_m,
                                      uint64_t az_looks, uint64_t rg_looks, float *coh, float *phase) {
  if (az_looks == 0 || rg_looks == 0) return SD_ERR_INSAR_INVALID_WINDOW_SIZE;
  const uint64_t n = lines * samples;
  const double c_light = 299792458.0;
  const double dtau = 2.0 * rps_m / c_light, off = (double)col_off;
  const double k = 6.283185307179586 / wavelength_m;
  std::vector<float> fe(n);
  for (uint64_t l = 0; l < lines; ++l) {
    const int64_t t = first_us + (int64_t)((double)l * ati * 1e6);
    double pr[3], vr[3], ps[3], vs[3], acc[3];
    if (orc_interpolate_orbit_and_accel(ref_svs, n_ref, t, pr, vr, acc) != 0) return SD_ERR_INSAR_ORBIT;
    if (orc_interpolate_orbit_and_accel(sec_svs, n_sec, t, ps, vs, acc) != 0) return SD_ERR_INSAR_ORBIT;
    for (uint64_t c = 0; c < samples; ++c) {
      const double tau = srt + ((double)c + off) * dtau;
      const double r_ref = tau * c_light / 2.0;
      double p[3];
      if (orc_ecef_from_slant_range_doppler(pr, vr, r_ref, 10, 1.0, p) != 0) {
        fe[l * samples + c] = 0.0f;
        continue;
      }
      const double dx = ps[0] - p[0], dy = ps[1] - p[1], dz = ps[2] - p[2];
      const double r_sec = std::sqrt(dx * dx + dy * dy + dz * dz);
      fe[l * samples + c] = (float)(k * 2.0 * (r_ref - r_sec));
    }
  }
  std::vector<float> ig_re(n), ig_im(n), rp(n), sp(n);
  for (uint64_t i = 0; i < n; ++i) {
    const float ri = ref[2 * i], rq = ref[2 * i + 1], si = sec[2 * i], sq = sec[2 * i + 1];
    const double phi = (double)fe[i];
    const double sn = std::sin(phi), cs = std::cos(phi);
    const double re = (double)si * cs + (double)sq * sn;
    const double im = (double)si * sn - (double)sq * cs;
    ig_re[i] = (float)((double)ri * re - (double)rq * im);
    ig_im[i] = (float)((double)ri * im + (double)rq * re);
    rp[i] = ri * ri + rq * rq;
    sp[i] = si * si + sq * sq;
  }
  const uint64_t ah = az_looks / 2, rh = rg_looks / 2;
  for (uint64_t l = 0; l < lines; ++l) {
    const uint64_t l0 = l > ah ? l - ah : 0, l1 = std::min(l + ah + 1, lines);
    for (uint64_t c = 0; c < samples; ++c) {
      const uint64_t c0 = c > rh ? c - rh : 0, c1 = std::min(c + rh + 1, samples);
      double sre = 0.0, sim = 0.0, srp = 0.0, ssp = 0.0;
      for (uint64_t wl = l0; wl < l1; ++wl)
        for (uint64_t wc = c0; wc < c1; ++wc) {
          const uint64_t w = wl * samples + wc;
          sre += (double)ig_re[w];
          sim += (double)ig_im[w];
          srp += (double)rp[w];
          ssp += (double)sp[w];
        }
      const double den = std::sqrt(srp * ssp);
      coh[l * samples + c] = den > 0.0 ? (float)std::fmin(std::sqrt(sre * sre + sim * sim) / den, 1.0) : 0.0f;
      if (phase) phase[l * samples + c] = (float)std::atan2(sim, sre);
    }
  }
  return SD_OK;
}

// compute_coreg_offsets (coreg.rs:128-223): the sparse grid in order, then
// fit_poly6 (478-517) with gaussian_elimination (522-568).
extern "C" int orc_solve_zero_doppler(const double *target, const sd_state_vector *svs, uint64_t n, int64_t guess,
                                      uint64_t max_iter, double tol, int64_t *t_out, int32_t *iters_out,
                                      double *residual_out);

extern "C" int orc_fit_poly6(const double *pts, uint64_t n, int which, double *coef, double *rms) {
  double a[6][6] = {}, b[6] = {};
  for (uint64_t p = 0; p < n; ++p) {
    const double l = pts[4 * p], c = pts[4 * p + 1], y = pts[4 * p + which];
    const double bs[6] = {1.0, l, c, l * l, l * c, c * c};
    for (int i = 0; i < 6; ++i) {
      b[i] += bs[i] * y;
      for (int j = 0; j < 6; ++j) a[i][j] += bs[i] * bs[j];
    }
  }
  for (int col = 0; col < 6; ++col) {
    int piv = col;  // Iterator::max_by keeps the last of equal maxima
    for (int r = col + 1; r < 6; ++r)
      if (std::fabs(a[r][col]) >= std::fabs(a[piv][col])) piv = r;
    for (int k = 0; k < 6; ++k) std::swap(a[col][k], a[piv][k]);
    std::swap(b[col], b[piv]);
    if (std::fabs(a[col][col]) < 1e-12) return SD_ERR_INSAR_COREG_GRID_TOO_SMALL;
    const double inv = 1.0 / a[col][col];
    for (int r = col + 1; r < 6; ++r) {
      const double f = a[r][col] * inv;
      for (int k = col; k < 6; ++k) a[r][k] -= f * a[col][k];
      b[r] -= f * b[col];
    }
  }
  for (int i = 5; i >= 0; --i) {
    double sum = b[i];
    for (int j = i + 1; j < 6; ++j) sum -= a[i][j] * coef[j];
    coef[i] = sum / a[i][i];
  }
  double sse = 0.0;
  for (uint64_t p = 0; p < n; ++p) {
    const double l = pts[4 * p], c = pts[4 * p + 1], y = pts[4 * p + which];
    const double res = y - orc_poly6(coef, l, c);
    sse += res * res;
  }
  *rms = std::sqrt(sse / (double)n);
  return SD_OK;
}

extern "C" int orc_coreg_offsets(const sd_state_vector *ro, uint64_t nr, int64_t ref_first, uint64_t lines,
                                 uint64_t samples, uint64_t ref_off, double ref_ati, double ref_tau0, double ref_rps,
                                 const sd_state_vector *so, uint64_t ns, int64_t sec_first, double sec_ati,
                                 double sec_tau0, double sec_rps, uint64_t sec_first_sample, double *az, double *rg,
                                 double *rms, uint64_t *n_valid) {
  const double c_light = 299792458.0;
  const double ref_dtau = 2.0 * ref_rps / c_light, sec_dtau = 2.0 * sec_rps / c_light;
  const double az_step = (double)lines / 21.0, rg_step = (double)samples / 51.0;
  std::vector<double> pts;
  for (int gi = 0; gi < 20; ++gi) {
    const double l = (double)(gi + 1) * az_step;
    for (int gj = 0; gj < 50; ++gj) {
      const double c = (double)(gj + 1) * rg_step;
      const int64_t t_ref = ref_first + (int64_t)(l * ref_ati * 1e6);
      const double range_m = (ref_tau0 + (c + (double)ref_off) * ref_dtau) * c_light / 2.0;
      double pos[3], vel[3], acc[3], P[3];
      if (orc_interpolate_orbit_and_accel(ro, nr, t_ref, pos, vel, acc) != 0) continue;
      if (orc_ecef_from_slant_range_doppler(pos, vel, range_m, 20, 1e-3, P) != 0) continue;
      int64_t t;
      int32_t it;
      double resid;
      if (orc_solve_zero_doppler(P, so, ns, sec_first, 20, 1e-9, &t, &it, &resid) != 0) continue;
      double sp[3], sv[3], sa[3];
      if (orc_interpolate_orbit_and_accel(so, ns, t, sp, sv, sa) != 0) continue;
      const double l_sec = (double)(t - sec_first) / (sec_ati * 1e6);
      const double rng = std::sqrt((P[0] - sp[0]) * (P[0] - sp[0]) + (P[1] - sp[1]) * (P[1] - sp[1]) +
                                   (P[2] - sp[2]) * (P[2] - sp[2]));
      const double c_sec = (2.0 * rng / c_light - sec_tau0) / sec_dtau - (double)sec_first_sample;
      pts.insert(pts.end(), {l, c, l_sec - l, c_sec - c});
    }
  }
  const uint64_t n = pts.size() / 4;
  *n_valid = n;
  if (n < 6) return SD_ERR_INSAR_COREG_GRID_TOO_SMALL;
  double ra, rr;
  if (orc_fit_poly6(pts.data(), n, 2, az, &ra) || orc_fit_poly6(pts.data(), n, 3, rg, &rr)) {
    *n_valid = 0;
    return SD_ERR_INSAR_COREG_GRID_TOO_SMALL;
  }
  *rms = std::sqrt((ra * ra + rr * rr) / 2.0);
  return SD_OK;
}
