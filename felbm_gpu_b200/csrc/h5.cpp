// HDF5 files from the published file-format specification (superblock
// version 0, version-1 object headers, symbol-table group). See h5.hpp.
#include "h5.hpp"

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
  // dataset object headers, then the data
  std::vector<std::vector<Msg>> hdrs(sets.size());
  std::vector<uint64_t> hdr_at(sets.size()), data_at(sets.size()), data_len(sets.size());
  uint64_t p = snod + snod_size;
  for (size_t q = 0; q < sets.size(); ++q) {
    const Dataset& d = sets[q];
    uint64_t count = 1;
    for (uint64_t x : d.dims) count *= x;
    data_len[q] = count * elem_size(d.type);
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
    Buf ly;                              // layout, version 3, contiguous (address set below)
    ly.u8(0, 3);
    ly.u8(1, 1);
    ly.at(18);
    hdrs[q] = {{0x0001, 0, ds.b}, {0x0003, 1, datatype(d.type)}, {0x0005, 1, fv.b}, {0x0008, 0, ly.b}};
    hdr_at[q] = p;
    p = pad8(p + header_size(hdrs[q]));
  }
  for (size_t q = 0; q < sets.size(); ++q) {
    data_at[q] = p;
    p = pad8(p + data_len[q]);
    Buf ly;
    ly.u8(0, 3);
    ly.u8(1, 1);
    ly.u64(2, data_len[q] ? data_at[q] : UNDEF);
    ly.u64(10, data_len[q]);
    hdrs[q][3].body = ly.b;
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
    f.bytes(data_at[q], sets[q].data, data_len[q]);
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
      uint64_t p = oh + 16, addr = UNDEF, len = 0;
      bool have_type = false;
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
        } else if (type == 0x0008) {
          if (f.b[d] != 3 || f.b[d + 1] != 1)
            return fe_fail(FE_ERR_IO, path + ": only contiguous datasets are supported (" + r.name + ")");
          addr = f.get(d + 2, 8);
          len = f.get(d + 10, 8);
        }
        p = d + msz;
      }
      uint64_t count = r.dims.empty() ? 0 : 1;
      for (uint64_t x : r.dims) count *= x;
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
