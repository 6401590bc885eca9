// HDF5 files from the published file-format specification (superblock
// version 0, version-1 object headers, symbol-table group). See h5.hpp.
#include "h5.hpp"

#include <zlib.h>

#include <algorithm>
#include <cstdio>
#include <cstring>

#include "../../include/felbm_b200.h"
#include "fe_internal.hpp"

namespace fe {
namespace h5 {
namespace {

constexpr uint64_t UNDEF = ~0ull;     // undefined address
constexpr int LEAF_K = 8;             // symbol-table node: 2K = 16 entries
constexpr int INTERNAL_K = 16;        // group B-tree node: 2K = 32 children
constexpr uint64_t HEAP_FREE_NONE = 1;  // "no free block" in a local heap (offsets are 8-aligned)
constexpr int ISTORE_K = 32;          // chunk B-tree node: 2K = 64 children (superblock 0 default)
constexpr unsigned FILTER_DEFLATE = 1;

uint64_t pad8(uint64_t x) { return (x + 7) & ~7ull; }
size_t elem_size(Type t) { return t == F64 ? 8 : 4; }

struct Buf {
  std::vector<unsigned char> b;
  void at(uint64_t off) {
    if (b.size() < off) b.resize(off, 0);
  }
  void u8(uint64_t off, unsigned v) { at(off + 1); b[off] = (unsigned char)v; }
  void u16(uint64_t off, unsigned v) { at(off + 2); for (int q = 0; q < 2; ++q) b[off + q] = (unsigned char)(v >> (8 * q)); }
  void u32(uint64_t off, uint64_t v) { at(off + 4); for (int q = 0; q < 4; ++q) b[off + q] = (unsigned char)(v >> (8 * q)); }
  void u64(uint64_t off, uint64_t v) { at(off + 8); for (int q = 0; q < 8; ++q) b[off + q] = (unsigned char)(v >> (8 * q)); }
  void bytes(uint64_t off, const void* p, size_t n) {
    at(off + n);
    if (n) std::memcpy(&b[off], p, n);
  }
};

// Datatype message body (class, bit fields, size, properties).
std::vector<unsigned char> datatype(Type t) {
  Buf m;
  if (t == F64 || t == F32) {
    const bool d = t == F64;
    m.u8(0, (1u << 4) | 1u);            // version 1, floating point
    m.u8(1, 0x20);                      // little endian, mantissa normalised (implied bit)
    m.u8(2, d ? 63 : 31);               // sign bit position
    m.u8(3, 0);
    m.u32(4, d ? 8 : 4);                // size
    m.u16(8, 0);                        // bit offset
    m.u16(10, d ? 64 : 32);             // precision
    m.u8(12, d ? 52 : 23);              // exponent location
    m.u8(13, d ? 11 : 8);               // exponent size
    m.u8(14, 0);                        // mantissa location
    m.u8(15, d ? 52 : 23);              // mantissa size
    m.u32(16, d ? 1023 : 127);          // exponent bias
  } else {
    m.u8(0, (1u << 4) | 0u);            // version 1, fixed point
    m.u8(1, t == I32 ? 0x08 : 0x00);    // little endian, signed for I32
    m.u8(2, 0);
    m.u8(3, 0);
    m.u32(4, 4);
    m.u16(8, 0);
    m.u16(10, 32);
  }
  return m.b;
}

// A version-1 object header with the given messages (type, flags, body).
struct Msg {
  unsigned type, flags;
  std::vector<unsigned char> body;
};
uint64_t header_size(const std::vector<Msg>& ms) {
  uint64_t s = 16;
  for (const Msg& m : ms) s += 8 + pad8(m.body.size());
  return s;
}
void put_header(Buf& f, uint64_t off, const std::vector<Msg>& ms) {
  f.u8(off, 1);                         // version
  f.u8(off + 1, 0);
  f.u16(off + 2, (unsigned)ms.size());  // messages
  f.u32(off + 4, 1);                    // reference count
  f.u32(off + 8, header_size(ms) - 16); // header data size
  uint64_t p = off + 16;                // messages start 8-aligned
  for (const Msg& m : ms) {
    const uint64_t sz = pad8(m.body.size());
    f.u16(p, m.type);
    f.u16(p + 2, (unsigned)sz);
    f.u8(p + 4, m.flags);
    f.bytes(p + 8, m.body.data(), m.body.size());
    f.at(p + 8 + sz);
    p += 8 + sz;
  }
}

}  // namespace

int write(const std::string& path, const std::vector<Dataset>& sets_in) {
  if (sets_in.empty() || sets_in.size() > 2 * LEAF_K) return fe_fail(FE_ERR_ARG, "hdf5 writer: 1..16 datasets");
  std::vector<Dataset> sets = sets_in;  // symbol-table entries are sorted by name
  std::sort(sets.begin(), sets.end(), [](const Dataset& a, const Dataset& b) { return a.name < b.name; });
  for (size_t q = 0; q < sets.size(); ++q) {
    if (sets[q].dims.empty() || sets[q].dims.size() > 2 || sets[q].name.empty())
      return fe_fail(FE_ERR_ARG, "hdf5 writer: 1-D or 2-D named datasets");
    if (q && sets[q].name == sets[q - 1].name) return fe_fail(FE_ERR_ARG, "hdf5 writer: duplicate dataset name");
  }
  // local heap: "" at offset 0, then the names
  std::vector<uint64_t> name_off;
  uint64_t heap_size = 8;
  for (const Dataset& d : sets) {
    name_off.push_back(heap_size);
    heap_size += pad8(d.name.size() + 1);
  }
  const uint64_t sb = 0, root = 96, heap = root + 40, heap_data = heap + 32;
  const uint64_t btree = pad8(heap_data + heap_size);
  const uint64_t btree_size = 24 + (2 * INTERNAL_K + 1) * 8 + 2 * INTERNAL_K * 8;
  const uint64_t snod = btree + btree_size;
  const uint64_t snod_size = 8 + 2 * LEAF_K * 40;
  // dataset object headers, then the data (chunked datasets: the chunk
  // B-tree node, then the compressed chunk)
  std::vector<std::vector<Msg>> hdrs(sets.size());
  std::vector<uint64_t> hdr_at(sets.size()), data_at(sets.size()), data_len(sets.size()), bt_at(sets.size(), 0);
  std::vector<std::vector<unsigned char>> packed(sets.size());
  uint64_t p = snod + snod_size;
  for (size_t q = 0; q < sets.size(); ++q) {
    const Dataset& d = sets[q];
    uint64_t count = 1;
    for (uint64_t x : d.dims) count *= x;
    data_len[q] = count * elem_size(d.type);
    if (d.deflate < 0 || d.deflate > 9) return fe_fail(FE_ERR_ARG, "hdf5 writer: deflate level 0-9");
    const bool chunked = d.deflate > 0 && count > 0;
    if (chunked) {
      if (data_len[q] >= (1ull << 32)) return fe_fail(FE_ERR_ARG, "hdf5 writer: a chunk is limited to 4 GB");
      uLongf clen = compressBound((uLong)data_len[q]);
      packed[q].resize(clen);
      if (compress2(packed[q].data(), &clen, static_cast<const Bytef*>(d.data), (uLong)data_len[q], d.deflate) != Z_OK)
        return fe_fail(FE_ERR_IO, "hdf5 writer: deflate failed");
      packed[q].resize(clen);
      data_len[q] = clen;
    }
    Buf ds;                              // dataspace, version 1
    ds.u8(0, 1);
    ds.u8(1, (unsigned)d.dims.size());
    ds.u8(2, 0);
    ds.at(8);
    for (size_t a = 0; a < d.dims.size(); ++a) ds.u64(8 + 8 * a, d.dims[a]);
    Buf fv;                              // fill value, version 2: none defined
    fv.u8(0, 2);
    fv.u8(1, 1);                         // space allocated early
    fv.u8(2, 2);                         // fill value never written
    fv.u8(3, 0);
    Buf ly;                              // layout, version 3 (addresses set below)
    ly.u8(0, 3);
    if (chunked) {
      ly.u8(1, 2);                       // chunked
      ly.u8(2, (unsigned)d.dims.size() + 1);
      ly.at(11 + 4 * (d.dims.size() + 1));
    } else {
      ly.u8(1, 1);                       // contiguous
      ly.at(18);
    }
    hdrs[q] = {{0x0001, 0, ds.b}, {0x0003, 1, datatype(d.type)}, {0x0005, 1, fv.b}};
    if (chunked) {
      Buf fp;                            // filter pipeline, version 1: deflate(level)
      fp.u8(0, 1);
      fp.u8(1, 1);
      fp.at(8);
      fp.u16(8, FILTER_DEFLATE);
      fp.u16(10, 0);                     // no name
      fp.u16(12, 0);                     // flags: mandatory
      fp.u16(14, 1);                     // one client value
      fp.u32(16, (unsigned)d.deflate);
      fp.at(24);                         // padded to an even number of values
      hdrs[q].push_back({0x000B, 1, fp.b});
    }
    hdrs[q].push_back({0x0008, 0, ly.b});
    hdr_at[q] = p;
    p = pad8(p + header_size(hdrs[q]));
  }
  auto bt_size = [&](size_t rank) {
    const uint64_t key = 8 + 8 * (rank + 1);
    return 24 + (2 * ISTORE_K + 1) * key + 2 * ISTORE_K * 8;
  };
  for (size_t q = 0; q < sets.size(); ++q) {
    if (!packed[q].empty()) {
      bt_at[q] = p;
      p = pad8(p + bt_size(sets[q].dims.size()));
    }
    data_at[q] = p;
    p = pad8(p + data_len[q]);
    Buf ly;
    ly.u8(0, 3);
    if (!packed[q].empty()) {
      const size_t rank = sets[q].dims.size();
      ly.u8(1, 2);
      ly.u8(2, (unsigned)rank + 1);
      ly.u64(3, bt_at[q]);
      for (size_t a = 0; a < rank; ++a) ly.u32(11 + 4 * a, (uint32_t)sets[q].dims[a]);  // one chunk
      ly.u32(11 + 4 * rank, (uint32_t)elem_size(sets[q].type));
    } else {
      ly.u8(1, 1);
      ly.u64(2, data_len[q] ? data_at[q] : UNDEF);
      ly.u64(10, data_len[q]);
    }
    hdrs[q].back().body = ly.b;
  }
  const uint64_t eof = p;

  Buf f;
  f.at(eof);
  // superblock version 0
  const unsigned char sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  f.bytes(sb, sig, 8);
  f.u8(8, 0);  f.u8(9, 0);  f.u8(10, 0);  f.u8(11, 0);  f.u8(12, 0);
  f.u8(13, 8); f.u8(14, 8); f.u8(15, 0);
  f.u16(16, LEAF_K);
  f.u16(18, INTERNAL_K);
  f.u32(20, 0);
  f.u64(24, 0);                          // base address
  f.u64(32, UNDEF);                      // free-space info
  f.u64(40, eof);                        // end of file
  f.u64(48, UNDEF);                      // driver information
  // root group symbol-table entry: cached B-tree and heap addresses
  f.u64(56, 0);
  f.u64(64, root);
  f.u32(72, 1);
  f.u32(76, 0);
  f.u64(80, btree);
  f.u64(88, heap);
  // root object header: one symbol-table message
  {
    Buf st;
    st.u64(0, btree);
    st.u64(8, heap);
    put_header(f, root, {{0x0011, 0, st.b}});
  }
  // local heap
  f.bytes(heap, "HEAP", 4);
  f.u8(heap + 4, 0);
  f.u64(heap + 8, heap_size);
  f.u64(heap + 16, HEAP_FREE_NONE);
  f.u64(heap + 24, heap_data);
  for (size_t q = 0; q < sets.size(); ++q)
    f.bytes(heap_data + name_off[q], sets[q].name.c_str(), sets[q].name.size() + 1);
  f.at(heap_data + heap_size);
  // B-tree: one leaf child (the symbol-table node); keys "" and the last name
  f.bytes(btree, "TREE", 4);
  f.u8(btree + 4, 0);
  f.u8(btree + 5, 0);
  f.u16(btree + 6, 1);
  f.u64(btree + 8, UNDEF);
  f.u64(btree + 16, UNDEF);
  f.u64(btree + 24, 0);
  f.u64(btree + 32, snod);
  f.u64(btree + 40, name_off.back());
  f.at(btree + btree_size);
  // symbol-table node
  f.bytes(snod, "SNOD", 4);
  f.u8(snod + 4, 1);
  f.u16(snod + 6, (unsigned)sets.size());
  for (size_t q = 0; q < sets.size(); ++q) {
    const uint64_t e = snod + 8 + 40 * q;
    f.u64(e, name_off[q]);
    f.u64(e + 8, hdr_at[q]);
    f.u32(e + 16, 0);
  }
  f.at(snod + snod_size);
  for (size_t q = 0; q < sets.size(); ++q) {
    put_header(f, hdr_at[q], hdrs[q]);
    if (packed[q].empty()) {
      f.bytes(data_at[q], sets[q].data, data_len[q]);
      continue;
    }
    // chunk B-tree (node type 1, leaf): key 0 = the chunk (stored size,
    // filter mask, offset 0 per axis), its address, then the bounding key
    const size_t rank = sets[q].dims.size();
    const uint64_t b = bt_at[q], key = 8 + 8 * (rank + 1);
    f.bytes(b, "TREE", 4);
    f.u8(b + 4, 1);
    f.u8(b + 5, 0);
    f.u16(b + 6, 1);
    f.u64(b + 8, UNDEF);
    f.u64(b + 16, UNDEF);
    f.u32(b + 24, (uint32_t)data_len[q]);
    f.u32(b + 28, 0);
    for (size_t a = 0; a <= rank; ++a) f.u64(b + 32 + 8 * a, 0);
    f.u64(b + 24 + key, data_at[q]);
    const uint64_t k1 = b + 24 + key + 8;
    f.u32(k1, 0);
    f.u32(k1 + 4, 0);
    for (size_t a = 0; a < rank; ++a) f.u64(k1 + 8 + 8 * a, sets[q].dims[a]);
    f.u64(k1 + 8 + 8 * rank, 0);
    f.at(b + bt_size(rank));
    f.bytes(data_at[q], packed[q].data(), packed[q].size());
  }
  f.at(eof);
  FILE* fp = std::fopen(path.c_str(), "wb");
  if (!fp) return fe_fail(FE_ERR_IO, "cannot open " + path + " for writing");
  const size_t w = std::fwrite(f.b.data(), 1, f.b.size(), fp);
  const int c = std::fclose(fp);
  if (w != f.b.size() || c != 0) return fe_fail(FE_ERR_IO, "short write to " + path);
  return FE_OK;
}

namespace {
struct In {
  std::vector<unsigned char> b;
  bool ok = true;
  uint64_t get(uint64_t off, int n) {
    if (off + n > b.size()) {
      ok = false;
      return 0;
    }
    uint64_t v = 0;
    for (int q = 0; q < n; ++q) v |= (uint64_t)b[off + q] << (8 * q);
    return v;
  }
};
}  // namespace

int read(const std::string& path, std::vector<Read>& out) {
  out.clear();
  In f;
  FILE* fp = std::fopen(path.c_str(), "rb");
  if (!fp) return fe_fail(FE_ERR_IO, "cannot open " + path);
  std::fseek(fp, 0, SEEK_END);
  const long sz = std::ftell(fp);
  std::fseek(fp, 0, SEEK_SET);
  f.b.resize(sz > 0 ? (size_t)sz : 0);
  const size_t got = f.b.empty() ? 0 : std::fread(f.b.data(), 1, f.b.size(), fp);
  std::fclose(fp);
  const unsigned char sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  if (got != f.b.size() || f.b.size() < 96 || std::memcmp(f.b.data(), sig, 8) != 0 || f.b[8] != 0 ||
      f.b[13] != 8 || f.b[14] != 8)
    return fe_fail(FE_ERR_IO, path + ": not an HDF5 file of the supported form");
  const uint64_t btree = f.get(80, 8), heap = f.get(88, 8);
  if (f.get(72, 4) != 1 || std::memcmp(&f.b[heap], "HEAP", 4) != 0 ||
      std::memcmp(&f.b[btree], "TREE", 4) != 0)
    return fe_fail(FE_ERR_IO, path + ": root group is not a symbol table");
  const uint64_t heap_size = f.get(heap + 8, 8), heap_data = f.get(heap + 24, 8);
  const unsigned used = (unsigned)f.get(btree + 6, 2);
  if (f.b[btree + 5] != 0) return fe_fail(FE_ERR_IO, path + ": multi-level group B-tree not supported");
  for (unsigned c = 0; c < used; ++c) {
    const uint64_t snod = f.get(btree + 24 + 16 * c + 8, 8);
    if (!f.ok || snod + 8 > f.b.size() || std::memcmp(&f.b[snod], "SNOD", 4) != 0)
      return fe_fail(FE_ERR_IO, path + ": bad symbol-table node");
    const unsigned nsym = (unsigned)f.get(snod + 6, 2);
    for (unsigned s = 0; s < nsym; ++s) {
      const uint64_t e = snod + 8 + 40 * s;
      const uint64_t noff = f.get(e, 8), oh = f.get(e + 8, 8);
      if (!f.ok || noff >= heap_size) return fe_fail(FE_ERR_IO, path + ": bad link name");
      Read r;
      r.name = reinterpret_cast<const char*>(&f.b[heap_data + noff]);
      // version-1 object header: dataspace, datatype, layout
      const unsigned nmsg = (unsigned)f.get(oh + 2, 2);
      uint64_t p = oh + 16, addr = UNDEF, len = 0, btree_at = UNDEF;
      bool have_type = false, chunked = false, deflate = false;
      std::vector<uint64_t> cdims;
      for (unsigned m = 0; m < nmsg && f.ok; ++m) {
        const unsigned type = (unsigned)f.get(p, 2), msz = (unsigned)f.get(p + 2, 2);
        const uint64_t d = p + 8;
        if (type == 0x0001) {
          const unsigned rank = f.b[d + 1];
          const uint64_t dims_at = d + (f.b[d] == 1 ? 8 : 4);
          for (unsigned a = 0; a < rank; ++a) r.dims.push_back(f.get(dims_at + 8 * a, 8));
        } else if (type == 0x0003) {
          const unsigned cls = f.b[d] & 0x0f, size = (unsigned)f.get(d + 4, 4);
          if (cls == 1) r.type = size == 8 ? F64 : F32;
          else if (cls == 0 && size == 4) r.type = (f.b[d + 1] & 0x08) ? I32 : U32;
          else return fe_fail(FE_ERR_IO, path + ": unsupported datatype of " + r.name);
          have_type = true;
        } else if (type == 0x000B) {
          // filter pipeline: deflate alone
          const unsigned ver = f.b[d], nf = f.b[d + 1];
          uint64_t q = d + (ver == 1 ? 8 : 2);
          for (unsigned k = 0; k < nf && f.ok; ++k) {
            const unsigned id = (unsigned)f.get(q, 2);
            const unsigned nlen = (ver == 1 || id >= 256) ? (unsigned)f.get(q + 2, 2) : 0;
            const unsigned ncd = (unsigned)f.get(q + (ver == 1 || id >= 256 ? 6 : 4), 2);
            if (id != FILTER_DEFLATE)
              return fe_fail(FE_ERR_IO, path + ": filter " + std::to_string(id) + " not supported (" + r.name + ")");
            deflate = true;
            q += (ver == 1 || id >= 256 ? 8 : 6) + (ver == 1 ? pad8(nlen) : nlen) + 4 * ncd;
            if (ver == 1 && (ncd & 1)) q += 4;
          }
        } else if (type == 0x0008) {
          if (f.b[d] != 3 || (f.b[d + 1] != 1 && f.b[d + 1] != 2))
            return fe_fail(FE_ERR_IO, path + ": only contiguous or chunked datasets are supported (" + r.name + ")");
          if (f.b[d + 1] == 1) {
            addr = f.get(d + 2, 8);
            len = f.get(d + 10, 8);
          } else {
            chunked = true;
            const unsigned nd = f.b[d + 2];
            btree_at = f.get(d + 3, 8);
            for (unsigned a = 0; a < nd; ++a) cdims.push_back(f.get(d + 11 + 4 * a, 4));
          }
        }
        p = d + msz;
      }
      uint64_t count = r.dims.empty() ? 0 : 1;
      for (uint64_t x : r.dims) count *= x;
      if (chunked) {
        // one chunk covering the dataset (what write() makes), deflated
        bool one = have_type && cdims.size() == r.dims.size() + 1 && btree_at + 24 <= f.b.size();
        for (size_t a = 0; one && a < r.dims.size(); ++a) one = cdims[a] == r.dims[a];
        if (!one || !deflate || std::memcmp(&f.b[btree_at], "TREE", 4) != 0 || f.b[btree_at + 4] != 1 ||
            f.b[btree_at + 5] != 0 || f.get(btree_at + 6, 2) != 1)
          return fe_fail(FE_ERR_IO, path + ": chunked dataset " + r.name + " is not one deflated chunk");
        const uint64_t key = 8 + 8 * cdims.size();
        const uint64_t clen = f.get(btree_at + 24, 4), caddr = f.get(btree_at + 24 + key, 8);
        if (!f.ok || caddr + clen > f.b.size()) return fe_fail(FE_ERR_IO, path + ": bad chunk of " + r.name);
        r.bytes.resize(count * elem_size(r.type));
        uLongf got_len = (uLongf)r.bytes.size();
        if (uncompress(r.bytes.data(), &got_len, &f.b[caddr], (uLong)clen) != Z_OK || got_len != r.bytes.size())
          return fe_fail(FE_ERR_IO, path + ": inflate failed for " + r.name);
        out.push_back(std::move(r));
        continue;
      }
      if (!f.ok || !have_type || count * elem_size(r.type) != len || (len && addr + len > f.b.size()))
        return fe_fail(FE_ERR_IO, path + ": bad dataset " + r.name);
      if (len) r.bytes.assign(f.b.begin() + addr, f.b.begin() + addr + len);
      out.push_back(std::move(r));
    }
  }
  return FE_OK;
}

}  // namespace h5
}  // namespace fe
