// h5write.cpp -- own-code writer for the HDF5 map files HipFT produces.
//
// The reference writes maps with the HDF5 library (wrh5, src/hipft.f90:
// 6155-6351): dataset "Data" (float32 when output_single_precision, else
// float64) with the Fortran dimensions (n1[,n2[,n3]]), and one scale dataset
// per dimension ("dim1", "dim2", "dim3") made a dimension scale and attached
// to "Data" (h5DSset_scale_f, h5DSattach_scale_f, h5DSset_label_f).  No HDF5
// library exists in this build environment, so this file lays out the same
// objects in the same on-disk format the library uses for such files (the
// maps in the reference's testsuite inputs have exactly this structure):
//
//   superblock version 0; root group as a symbol table (v1 B-tree, local
//   heap, one symbol node); version-1 object headers; version-1 dataspaces;
//   IEEE little-endian float datatypes; fill-value message version 2;
//   contiguous layout (layout message version 3); attributes (message
//   version 1):
//     scales: CLASS = "DIMENSION_SCALE", NAME = "dimN", REFERENCE_LIST =
//             {object reference to "Data", dimension index};
//     Data:   DIMENSION_LIST (variable-length sequences of object references)
//             and DIMENSION_LABELS (variable-length strings), whose elements
//             live in one global heap collection.
//   Entry c of DIMENSION_LIST / DIMENSION_LABELS names scale "dim<c+1>", the
//   convention of the reference's own map files.
//
// Addresses are absolute (base address 0), offsets and lengths 8 bytes.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/hipft_gpu.h"

namespace {

constexpr uint64_t kUndef = ~0ull;
constexpr int kLeafK = 4, kIntK = 16;  // group B-tree leaf / internal K (library defaults)

struct Out {
  std::vector<uint8_t> b;
  size_t size() const { return b.size(); }
  void u8(unsigned v) { b.push_back((uint8_t)v); }
  void u16(unsigned v) { for (int i = 0; i < 2; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
  void u32(uint32_t v) { for (int i = 0; i < 4; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
  void u64(uint64_t v) { for (int i = 0; i < 8; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
  void raw(const void *p, size_t n) { b.insert(b.end(), (const uint8_t *)p, (const uint8_t *)p + n); }
  void zeros(size_t n) { b.insert(b.end(), n, 0); }
  void pad8() { while (b.size() % 8) b.push_back(0); }
  void put64(size_t at, uint64_t v) { for (int i = 0; i < 8; ++i) b[at + i] = (uint8_t)(v >> (8 * i)); }
};

// ------------------------------------------------------------- datatypes
std::vector<uint8_t> float_type(bool single) {
  Out o;
  o.u8(0x11);  // version 1, class 1 (floating point)
  o.u8(0x20);  // little endian, mantissa normalisation: implied leading 1
  o.u8(single ? 31 : 63);  // sign bit position
  o.u8(0);
  o.u32(single ? 4 : 8);
  o.u16(0);                 // bit offset
  o.u16(single ? 32 : 64);  // precision
  o.u8(single ? 23 : 52);   // exponent location
  o.u8(single ? 8 : 11);    // exponent size
  o.u8(0);                  // mantissa location
  o.u8(single ? 23 : 52);   // mantissa size
  o.u32(single ? 127 : 1023);
  return o.b;
}
std::vector<uint8_t> string_type(uint32_t n) {  // fixed length, NUL terminated, ASCII
  Out o;
  o.u8(0x13);
  o.u8(0);
  o.u8(0);
  o.u8(0);
  o.u32(n);
  return o.b;
}
std::vector<uint8_t> objref_type() {
  Out o;
  o.u8(0x17);  // version 1, class 7 (reference), object reference
  o.u8(0);
  o.u8(0);
  o.u8(0);
  o.u32(8);
  return o.b;
}
std::vector<uint8_t> vlen_objref_type() {
  Out o;
  o.u8(0x19);  // version 1, class 9 (variable length), sequence
  o.u8(0);
  o.u8(0);
  o.u8(0);
  o.u32(16);
  auto base = objref_type();
  o.raw(base.data(), base.size());
  return o.b;
}
std::vector<uint8_t> vlen_string_type() {
  Out o;
  o.u8(0x19);
  o.u8(0x01);  // string, NUL-terminated padding, ASCII
  o.u8(0);
  o.u8(0);
  o.u32(16);
  o.u8(0x10);  // base: 1-byte unsigned integer
  o.u8(0);
  o.u8(0);
  o.u8(0);
  o.u32(1);
  o.u16(0);
  o.u16(8);
  return o.b;
}
// compound {object reference "dataset"; int32 "dimension"} of 16 bytes
std::vector<uint8_t> reflist_type() {
  Out o;
  o.u8(0x16);  // version 1, class 6 (compound)
  o.u16(2);    // members
  o.u8(0);
  o.u32(16);
  auto member = [&](const char *name, uint32_t off, const std::vector<uint8_t> &t) {
    size_t n = std::strlen(name) + 1;
    o.raw(name, n);
    o.zeros((8 - n % 8) % 8);
    o.u32(off);
    o.u8(0);  // dimensionality
    o.zeros(3);
    o.u32(0);  // permutation
    o.u32(0);
    o.zeros(16);  // dimension sizes
    o.raw(t.data(), t.size());
  };
  member("dataset", 0, objref_type());
  Out i32;
  i32.u8(0x10);
  i32.u8(0x08);  // signed
  i32.u8(0);
  i32.u8(0);
  i32.u32(4);
  i32.u16(0);
  i32.u16(32);
  member("dimension", 8, i32.b);
  return o.b;
}

std::vector<uint8_t> simple_space(const std::vector<uint64_t> &dims) {  // version 1, with max dims
  Out o;
  o.u8(1);
  o.u8((unsigned)dims.size());
  o.u8(1);
  o.u8(0);
  o.u32(0);
  for (auto d : dims) o.u64(d);
  for (auto d : dims) o.u64(d);
  return o.b;
}
std::vector<uint8_t> scalar_space() {
  Out o;
  o.u8(1);
  o.u8(0);
  o.u8(0);
  o.u8(0);
  o.u32(0);
  return o.b;
}

std::vector<uint8_t> attribute(const char *name, const std::vector<uint8_t> &type,
                               const std::vector<uint8_t> &space, const std::vector<uint8_t> &data) {
  Out o;
  size_t nl = std::strlen(name) + 1;
  o.u8(1);
  o.u8(0);
  o.u16((unsigned)nl);
  o.u16((unsigned)type.size());
  o.u16((unsigned)space.size());
  o.raw(name, nl);
  o.pad8();
  o.raw(type.data(), type.size());
  o.pad8();
  o.raw(space.data(), space.size());
  o.pad8();
  o.raw(data.data(), data.size());
  o.pad8();
  return o.b;
}

struct Msg {
  unsigned type, flags;
  std::vector<uint8_t> body;  // padded to 8 on output
};

size_t header_size(const std::vector<Msg> &m) {
  size_t s = 0;
  for (auto &x : m) s += 8 + ((x.body.size() + 7) & ~size_t(7));
  return s;
}
void put_header(Out &o, const std::vector<Msg> &m) {
  o.u8(1);  // version
  o.u8(0);
  o.u16((unsigned)m.size());
  o.u32(1);  // reference count
  o.u32((uint32_t)header_size(m));
  o.u32(0);  // alignment
  for (auto &x : m) {
    size_t n = (x.body.size() + 7) & ~size_t(7);
    o.u16(x.type);
    o.u16((unsigned)n);
    o.u8(x.flags);
    o.zeros(3);
    o.raw(x.body.data(), x.body.size());
    o.zeros(n - x.body.size());
  }
}

std::vector<uint8_t> fill_msg() { return {2, 2, 2, 1, 0, 0, 0, 0}; }
std::vector<uint8_t> layout_msg(uint64_t addr, uint64_t size) {
  Out o;
  o.u8(3);
  o.u8(1);  // contiguous
  o.u64(addr);
  o.u64(size);
  return o.b;
}

}  // namespace

// Write a 1-3 dimensional map with scales as wrh5 does (src/hipft.f90:
// 6155-6351).  dims are Fortran dimensions (dims[0] varies fastest in
// `data`); s1..s3 the scales (all present for ndim dimensions).
extern "C" int hipft_h5_write(const char *path, int ndim, const int64_t dims[3], const double *data,
                              const double *s1, const double *s2, const double *s3, int single_precision) {
  if (!path || !dims || !data || ndim < 1 || ndim > 3) return HIPFT_EINVAL;
  const double *sc[3] = {s1, s2, s3};
  uint64_t n = 1;
  for (int i = 0; i < ndim; ++i) {
    if (dims[i] < 1 || !sc[i]) return HIPFT_EINVAL;
    n *= (uint64_t)dims[i];
  }
  const bool single = single_precision != 0;
  const uint64_t es = single ? 4 : 8;
  std::vector<uint64_t> cdims;  // C order: slowest first
  for (int i = ndim - 1; i >= 0; --i) cdims.push_back((uint64_t)dims[i]);

  // ---- fixed layout of the metadata
  const uint64_t a_root = 96, a_btree = 136;
  const uint64_t btree_size = 24 + (2 * kIntK + 1) * 8 + 2 * kIntK * 8;
  const uint64_t a_heap = a_btree + btree_size;
  // local heap data: "" at 0, "Data" at 8, "dimN" at 16 + 8(N-1), then one free block
  const uint64_t names_size = 16 + 8 * (uint64_t)ndim, heap_free = 16;
  const uint64_t a_heapdata = a_heap + 32;
  const uint64_t a_snod = a_heapdata + names_size + heap_free;
  const uint64_t snod_size = 8 + 2 * kLeafK * 40;
  const uint64_t a_data_oh = a_snod + snod_size;

  // object headers depend on addresses only through fixed-size fields, so
  // their sizes are computed with placeholder addresses first
  auto data_msgs = [&](uint64_t raw_addr, uint64_t gcol, uint32_t first_idx) {
    std::vector<Msg> m;
    m.push_back({0x0001, 0, simple_space(cdims)});
    m.push_back({0x0003, 1, float_type(single)});
    m.push_back({0x0005, 1, fill_msg()});
    m.push_back({0x0008, 1, layout_msg(raw_addr, n * es)});
    Out dl, lb;
    for (int c = 0; c < ndim; ++c) {
      dl.u32(1);
      dl.u64(gcol);
      dl.u32(first_idx + (uint32_t)c);
      lb.u32(4);
      lb.u64(gcol);
      lb.u32(first_idx + (uint32_t)ndim + (uint32_t)c);
    }
    std::vector<uint64_t> nd{(uint64_t)ndim};
    m.push_back({0x000C, 0, attribute("DIMENSION_LIST", vlen_objref_type(), simple_space(nd), dl.b)});
    m.push_back({0x000C, 0, attribute("DIMENSION_LABELS", vlen_string_type(), simple_space(nd), lb.b)});
    return m;
  };
  auto scale_msgs = [&](int i, uint64_t raw_addr, uint64_t data_oh) {
    std::vector<Msg> m;
    std::vector<uint64_t> d1{(uint64_t)dims[i]};
    m.push_back({0x0001, 0, simple_space(d1)});
    m.push_back({0x0003, 1, float_type(single)});
    m.push_back({0x0005, 1, fill_msg()});
    m.push_back({0x0008, 1, layout_msg(raw_addr, (uint64_t)dims[i] * es)});
    const char cls[16] = "DIMENSION_SCALE";
    m.push_back({0x000C, 0, attribute("CLASS", string_type(16), scalar_space(),
                                      std::vector<uint8_t>(cls, cls + 16))});
    char nm[5] = {'d', 'i', 'm', (char)('1' + i), 0};
    m.push_back({0x000C, 0, attribute("NAME", string_type(5), scalar_space(), std::vector<uint8_t>(nm, nm + 5))});
    Out rl;
    rl.u64(data_oh);
    rl.u32((uint32_t)i);  // index of this scale's entry in Data's DIMENSION_LIST
    rl.u32(0);
    std::vector<uint64_t> one{1};
    m.push_back({0x000C, 0, attribute("REFERENCE_LIST", reflist_type(), simple_space(one), rl.b)});
    return m;
  };
  const uint64_t data_oh_size = 16 + header_size(data_msgs(0, 0, 1));
  std::vector<uint64_t> a_scale_oh(ndim);
  uint64_t p = a_data_oh + data_oh_size;
  for (int i = 0; i < ndim; ++i) {
    a_scale_oh[i] = p;
    p += 16 + header_size(scale_msgs(i, 0, 0));
  }
  const uint64_t a_gcol = p, gcol_size = 4096;
  p += gcol_size;
  const uint64_t a_raw = p;
  std::vector<uint64_t> a_sraw(ndim);
  p += (n * es + 7) & ~uint64_t(7);
  for (int i = 0; i < ndim; ++i) {
    a_sraw[i] = p;
    p += ((uint64_t)dims[i] * es + 7) & ~uint64_t(7);
  }
  const uint64_t eof = p;

  Out o;
  o.b.reserve((size_t)eof);
  // ---- superblock (version 0)
  const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  o.raw(sig, 8);
  o.u8(0);  // superblock version
  o.u8(0);  // free-space version
  o.u8(0);  // root symbol table entry version
  o.u8(0);
  o.u8(0);  // shared header message version
  o.u8(8);  // size of offsets
  o.u8(8);  // size of lengths
  o.u8(0);
  o.u16(kLeafK);
  o.u16(kIntK);
  o.u32(0);  // consistency flags
  o.u64(0);  // base address
  o.u64(kUndef);  // free-space info
  o.u64(eof);
  o.u64(kUndef);  // driver info
  // root group symbol table entry: cache type 1 holds the B-tree and heap
  o.u64(0);
  o.u64(a_root);
  o.u32(1);
  o.u32(0);
  o.u64(a_btree);
  o.u64(a_heap);
  // ---- root object header: symbol table message
  {
    Out st;
    st.u64(a_btree);
    st.u64(a_heap);
    put_header(o, {{0x0011, 0, st.b}});
  }
  // ---- group B-tree: one leaf entry pointing at the symbol node
  if (o.size() != a_btree) return HIPFT_EIO;
  o.raw("TREE", 4);
  o.u8(0);  // group node
  o.u8(0);  // level
  o.u16(1);
  o.u64(kUndef);
  o.u64(kUndef);
  o.u64(0);                              // key 0: ""
  o.u64(a_snod);                         // child 0
  o.u64(16 + 8 * (uint64_t)(ndim - 1));  // key 1: the last name in the node
  o.zeros((size_t)(a_btree + btree_size - o.size()));
  // ---- local heap with the link names
  o.raw("HEAP", 4);
  o.u8(0);
  o.zeros(3);
  o.u64(names_size + heap_free);
  o.u64(names_size);  // head of the free list
  o.u64(a_heapdata);
  o.zeros(8);
  o.raw("Data", 4);
  o.zeros(4);
  for (int i = 0; i < ndim; ++i) {
    char nm[8] = {'d', 'i', 'm', (char)('1' + i), 0, 0, 0, 0};
    o.raw(nm, 8);
  }
  o.u64(1);  // free block: no next block
  o.u64(heap_free);
  // ---- symbol node: Data, dim1.. (sorted by name)
  if (o.size() != a_snod) return HIPFT_EIO;
  o.raw("SNOD", 4);
  o.u8(1);
  o.u8(0);
  o.u16((unsigned)(1 + ndim));
  auto entry = [&](uint64_t name_off, uint64_t oh) {
    o.u64(name_off);
    o.u64(oh);
    o.u32(0);
    o.u32(0);
    o.zeros(16);
  };
  entry(8, a_data_oh);
  for (int i = 0; i < ndim; ++i) entry(16 + 8 * (uint64_t)i, a_scale_oh[i]);
  o.zeros((size_t)(a_snod + snod_size - o.size()));
  // ---- dataset and scale object headers
  if (o.size() != a_data_oh) return HIPFT_EIO;
  put_header(o, data_msgs(a_raw, a_gcol, 1));
  for (int i = 0; i < ndim; ++i) {
    if (o.size() != a_scale_oh[i]) return HIPFT_EIO;
    put_header(o, scale_msgs(i, a_sraw[i], a_data_oh));
  }
  // ---- global heap: references to the scales, then their labels
  if (o.size() != a_gcol) return HIPFT_EIO;
  o.raw("GCOL", 4);
  o.u8(1);
  o.zeros(3);
  o.u64(gcol_size);
  uint16_t idx = 1;
  for (int i = 0; i < ndim; ++i, ++idx) {
    o.u16(idx);
    o.u16(0);
    o.u32(0);
    o.u64(8);
    o.u64(a_scale_oh[i]);
  }
  for (int i = 0; i < ndim; ++i, ++idx) {
    o.u16(idx);
    o.u16(0);
    o.u32(0);
    o.u64(4);
    char nm[8] = {'d', 'i', 'm', (char)('1' + i), 0, 0, 0, 0};
    o.raw(nm, 8);
  }
  const uint64_t used = o.size() - a_gcol;
  o.u16(0);  // free space object
  o.u16(0);
  o.u32(0);
  o.u64(gcol_size - used);
  o.zeros((size_t)(a_gcol + gcol_size - o.size()));
  // ---- raw data
  if (o.size() != a_raw) return HIPFT_EIO;
  auto put_values = [&](const double *v, uint64_t cnt) {
    if (single) {
      for (uint64_t q = 0; q < cnt; ++q) {
        float x = (float)v[q];
        o.raw(&x, 4);
      }
    } else {
      o.raw(v, cnt * 8);
    }
    o.pad8();
  };
  put_values(data, n);
  for (int i = 0; i < ndim; ++i) put_values(sc[i], (uint64_t)dims[i]);
  if (o.size() != eof) return HIPFT_EIO;

  FILE *fp = std::fopen(path, "wb");
  if (!fp) return HIPFT_EIO;
  const size_t wrote = std::fwrite(o.b.data(), 1, o.b.size(), fp);
  const int cl = std::fclose(fp);
  return (wrote == o.b.size() && cl == 0) ? HIPFT_OK : HIPFT_EIO;
}
