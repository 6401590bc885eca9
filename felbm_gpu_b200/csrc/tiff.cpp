// Segmented TIFF stacks for the reference's 3d_image geometry
// (cfg/3d_image/domain.cfg: image_dir, extension, interface_solid,
// invert_image, coarsening_levels, use_subvolume; its reader,
// DomainInitializer_3DImage, is in the absent felbm_local tree and links
// libtiff, which this image lacks). A baseline-TIFF reader written from the
// TIFF 6.0 specification (Adobe, 1992): both byte orders, every page of every
// file in the order given (one page = one z slice), grey images of 1, 8 or 16
// bits per sample, one sample per pixel, strips, no compression or PackBits.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/felbm_b200.h"
#include "fe_internal.hpp"

namespace {

struct Page {
  uint32_t w = 0, h = 0, bits = 1, spp = 1, comp = 1, planar = 1, rows_per_strip = 0xFFFFFFFFu;
  std::vector<uint64_t> offs, counts;
};

struct Reader {
  std::vector<uint8_t> b;
  bool be = false;  // big-endian ("MM")
  std::string name;
  std::string err;

  bool in(uint64_t off, uint64_t n) const { return off <= b.size() && n <= b.size() - off; }
  uint32_t u16(uint64_t o) const { return be ? (b[o] << 8) | b[o + 1] : b[o] | (b[o + 1] << 8); }
  uint32_t u32(uint64_t o) const {
    return be ? ((uint32_t)b[o] << 24) | ((uint32_t)b[o + 1] << 16) | ((uint32_t)b[o + 2] << 8) | b[o + 3]
              : b[o] | ((uint32_t)b[o + 1] << 8) | ((uint32_t)b[o + 2] << 16) | ((uint32_t)b[o + 3] << 24);
  }
  bool fail(const std::string& m) {
    err = name + ": " + m;
    return false;
  }
  // Values of a SHORT or LONG field (count entries), inline or at an offset.
  bool values(uint64_t entry, std::vector<uint64_t>& out) {
    const uint32_t type = u16(entry + 2), count = u32(entry + 4);
    const int size = type == 3 ? 2 : (type == 4 ? 4 : (type == 1 ? 1 : 0));
    if (!size) return fail("unsupported field type " + std::to_string(type));
    const uint64_t bytes = (uint64_t)size * count;
    const uint64_t at = bytes <= 4 ? entry + 8 : u32(entry + 8);
    if (!in(at, bytes)) return fail("field outside the file");
    out.resize(count);
    for (uint32_t k = 0; k < count; ++k)
      out[k] = size == 2 ? u16(at + 2 * k) : (size == 4 ? u32(at + 4 * k) : b[at + k]);
    return true;
  }
  bool pages(std::vector<Page>& out) {
    if (b.size() < 8) return fail("not a TIFF file");
    if (b[0] == 'I' && b[1] == 'I') be = false;
    else if (b[0] == 'M' && b[1] == 'M') be = true;
    else return fail("not a TIFF file");
    if (u16(2) != 42) return fail("not a TIFF file (BigTIFF is not supported)");
    uint64_t ifd = u32(4);
    int guard = 0;
    while (ifd) {
      if (++guard > 1000000 || !in(ifd, 2)) return fail("broken page chain");
      const uint32_t ne = u16(ifd);
      if (!in(ifd + 2, 12ull * ne + 4)) return fail("page directory outside the file");
      Page p;
      std::vector<uint64_t> v;
      for (uint32_t k = 0; k < ne; ++k) {
        const uint64_t e = ifd + 2 + 12ull * k;
        const uint32_t tag = u16(e);
        switch (tag) {
          case 256: case 257: case 258: case 259: case 277: case 278: case 284: case 273: case 279:
            if (!values(e, v) || v.empty()) return err.empty() ? fail("empty field") : false;
            break;
          default:
            continue;
        }
        if (tag == 256) p.w = (uint32_t)v[0];
        else if (tag == 257) p.h = (uint32_t)v[0];
        else if (tag == 258) p.bits = (uint32_t)v[0];
        else if (tag == 259) p.comp = (uint32_t)v[0];
        else if (tag == 277) p.spp = (uint32_t)v[0];
        else if (tag == 278) p.rows_per_strip = (uint32_t)v[0];
        else if (tag == 284) p.planar = (uint32_t)v[0];
        else if (tag == 273) p.offs = v;
        else p.counts = v;
      }
      if (!p.w || !p.h) return fail("page without width or height");
      if (p.spp != 1) return fail("only one sample per pixel (grey) is supported");
      if (p.bits != 1 && p.bits != 8 && p.bits != 16) return fail("bits per sample must be 1, 8 or 16");
      if (p.comp != 1 && p.comp != 32773) return fail("unsupported compression " + std::to_string(p.comp) +
                                                      " (uncompressed and PackBits are read)");
      if (p.offs.empty() || p.offs.size() != p.counts.size()) return fail("strips missing");
      out.push_back(std::move(p));
      ifd = u32(ifd + 2 + 12ull * ne);
    }
    return true;
  }
  // The page's pixels as 0/nonzero flags (w*h), rows top to bottom.
  bool pixels(const Page& p, std::vector<uint8_t>& out) {
    const uint64_t row_bytes = p.bits == 1 ? (p.w + 7) / 8 : (uint64_t)p.w * (p.bits / 8);
    std::vector<uint8_t> raw;
    raw.reserve(row_bytes * p.h);
    for (size_t s = 0; s < p.offs.size(); ++s) {
      if (!in(p.offs[s], p.counts[s])) return fail("strip outside the file");
      const uint8_t* src = b.data() + p.offs[s];
      if (p.comp == 1) {
        raw.insert(raw.end(), src, src + p.counts[s]);
      } else {  // PackBits: n >= 0 copies n+1 bytes, n in [-127,-1] repeats the next byte 1-n times
        uint64_t k = 0;
        while (k < p.counts[s]) {
          const int8_t n = (int8_t)src[k++];
          if (n >= 0) {
            if (k + n + 1 > p.counts[s]) return fail("PackBits run outside the strip");
            raw.insert(raw.end(), src + k, src + k + n + 1);
            k += n + 1;
          } else if (n != -128) {
            if (k >= p.counts[s]) return fail("PackBits run outside the strip");
            raw.insert(raw.end(), (size_t)(1 - n), src[k++]);
          }
        }
      }
    }
    if (raw.size() < row_bytes * p.h) return fail("fewer pixel bytes than the page needs");
    out.assign((size_t)p.w * p.h, 0);
    for (uint32_t y = 0; y < p.h; ++y) {
      const uint8_t* r = raw.data() + y * row_bytes;
      for (uint32_t x = 0; x < p.w; ++x) {
        uint32_t v;
        if (p.bits == 1) v = (r[x >> 3] >> (7 - (x & 7))) & 1u;
        else if (p.bits == 8) v = r[x];
        else v = r[2 * x] | r[2 * x + 1];  // nonzero either way round
        out[(size_t)y * p.w + x] = v != 0;
      }
    }
    return true;
  }
};

}  // namespace

extern "C" {

int fe_geom_tiff_stack(const char* const* paths, int npaths, int solid_nonzero, int invert, int coarsening_levels,
                       const int* subvolume, int* dims, uint8_t* solid, int64_t capacity) {
  if (!paths || npaths < 1 || !dims || coarsening_levels < 0 || coarsening_levels > 16)
    return fe_fail(FE_ERR_ARG, "fe_geom_tiff_stack: bad arguments");
  // full-resolution stack, z = page index over the files in order
  std::vector<uint8_t> full;
  int64_t W = -1, H = -1, D = 0;
  for (int f = 0; f < npaths; ++f) {
    Reader rd;
    rd.name = paths[f] ? paths[f] : "";
    FILE* fp = std::fopen(rd.name.c_str(), "rb");
    if (!fp) return fe_fail(FE_ERR_IO, "cannot open " + rd.name);
    std::fseek(fp, 0, SEEK_END);
    const long size = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    rd.b.resize(size > 0 ? (size_t)size : 0);
    const size_t got = rd.b.empty() ? 0 : std::fread(rd.b.data(), 1, rd.b.size(), fp);
    std::fclose(fp);
    if (got != rd.b.size()) return fe_fail(FE_ERR_IO, "short read of " + rd.name);
    std::vector<Page> pages;
    if (!rd.pages(pages)) return fe_fail(FE_ERR_IO, rd.err);
    for (const Page& p : pages) {
      if (W < 0) {
        W = p.w;
        H = p.h;
      } else if (p.w != W || p.h != H) {
        return fe_fail(FE_ERR_ARG, rd.name + ": page size differs from the stack's");
      }
      std::vector<uint8_t> px;
      if (!rd.pixels(p, px)) return fe_fail(FE_ERR_IO, rd.err);
      full.insert(full.end(), px.begin(), px.end());
      ++D;
    }
  }
  if (D == 0) return fe_fail(FE_ERR_ARG, "no page in the stack");
  // voxel rule: solid where the value is nonzero (interface_solid) or zero,
  // then inverted on request
  for (uint8_t& v : full) v = (uint8_t)((solid_nonzero ? v != 0 : v == 0) != (invert != 0));
  // sub-volume in full-resolution voxels
  int64_t x0 = 0, y0 = 0, z0 = 0, nx = W, ny = H, nz = D;
  if (subvolume) {
    x0 = subvolume[0]; y0 = subvolume[1]; z0 = subvolume[2];
    nx = subvolume[3]; ny = subvolume[4]; nz = subvolume[5];
    if (x0 < 0 || y0 < 0 || z0 < 0 || nx < 1 || ny < 1 || nz < 1 || x0 + nx > W || y0 + ny > H || z0 + nz > D)
      return fe_fail(FE_ERR_ARG, "sub-volume outside the image (" + std::to_string(W) + " x " + std::to_string(H) +
                                     " x " + std::to_string(D) + ")");
  }
  std::vector<uint8_t> cur((size_t)nx * ny * nz);
  for (int64_t z = 0; z < nz; ++z)
    for (int64_t y = 0; y < ny; ++y)
      std::memcpy(&cur[(size_t)((z * ny + y) * nx)], &full[(size_t)(((z0 + z) * H + (y0 + y)) * W + x0)], nx);
  full.clear();
  full.shrink_to_fit();
  // coarsening: each level halves every axis of extent > 1 (a trailing odd
  // layer is dropped); a coarse voxel is solid when at least half of its
  // fine voxels are
  for (int l = 0; l < coarsening_levels; ++l) {
    const int fx = nx > 1 ? 2 : 1, fy = ny > 1 ? 2 : 1, fz = nz > 1 ? 2 : 1;
    const int64_t cx = nx / fx, cy = ny / fy, cz = nz / fz;
    if (cx < 1 || cy < 1 || cz < 1) return fe_fail(FE_ERR_ARG, "coarsening leaves no voxel");
    const int cells = fx * fy * fz;
    std::vector<uint8_t> nxt((size_t)cx * cy * cz);
    for (int64_t z = 0; z < cz; ++z)
      for (int64_t y = 0; y < cy; ++y)
        for (int64_t x = 0; x < cx; ++x) {
          int s = 0;
          for (int dz = 0; dz < fz; ++dz)
            for (int dy = 0; dy < fy; ++dy)
              for (int dx = 0; dx < fx; ++dx) s += cur[(size_t)(((z * fz + dz) * ny + y * fy + dy) * nx + x * fx + dx)];
          nxt[(size_t)((z * cy + y) * cx + x)] = (uint8_t)(2 * s >= cells);
        }
    cur.swap(nxt);
    nx = cx; ny = cy; nz = cz;
  }
  if (nx > INT32_MAX || ny > INT32_MAX || nz > INT32_MAX) return fe_fail(FE_ERR_ARG, "image too large");
  dims[0] = (int)nx;
  dims[1] = (int)ny;
  dims[2] = (int)nz;
  if (solid) {
    if (capacity < (int64_t)cur.size()) return fe_fail(FE_ERR_ARG, "fe_geom_tiff_stack: mask buffer too small");
    std::memcpy(solid, cur.data(), cur.size());
  }
  return FE_OK;
}

}  // extern "C"
