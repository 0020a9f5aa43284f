// h5lite.cpp -- minimal reader for the HDF5 map files HipFT exchanges.
//
// The reference reads maps with the HDF5 library (rdh5, src/hipft.f90:5678):
// the first object of the root group ("Data") is the field and the remaining
// ones ("dim1", "dim2", "dim3") are its scales.  No HDF5 library exists in
// this build environment, so this file decodes the subset of the format
// those files use: superblock version 0 or 1, a root group stored as a
// symbol table (v1 B-tree + local heap + symbol nodes), version-1 object
// headers (with continuation blocks), simple dataspaces, IEEE float32/float64
// little-endian datatypes and contiguous or compact data layout.  Anything
// else is rejected with HIPFT_EIO rather than guessed at.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/hipft_gpu.h"

namespace {

struct H5File {
  std::vector<uint8_t> buf;
  int so = 8, sl = 8;  // size of offsets / lengths
  uint64_t base = 0;

  bool load(const char *path) {
    FILE *fp = std::fopen(path, "rb");
    if (!fp) return false;
    std::fseek(fp, 0, SEEK_END);
    long n = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    if (n <= 0) { std::fclose(fp); return false; }
    buf.resize((size_t)n);
    size_t got = std::fread(buf.data(), 1, (size_t)n, fp);
    std::fclose(fp);
    return got == (size_t)n;
  }
  bool in(uint64_t off, uint64_t len) const { return off <= buf.size() && len <= buf.size() - off; }
  uint64_t u(uint64_t off, int nbytes) const {
    uint64_t v = 0;
    for (int i = nbytes - 1; i >= 0; --i) v = (v << 8) | buf[off + i];
    return v;
  }
};

struct Dataset {
  std::vector<uint64_t> dims;  // C order (slowest first)
  int elsize = 0;
  int fclass = -1;
  bool little = true;
  int layout = -1;  // 0 compact, 1 contiguous
  uint64_t addr = 0, size = 0;
  uint64_t compact_off = 0;
};

// Parse the messages of a version-1 object header at `addr`.
bool parse_object(const H5File &F, uint64_t addr, Dataset &ds, uint64_t *btree, uint64_t *heap) {
  if (!F.in(addr, 16) || F.buf[addr] != 1) return false;
  uint32_t nmsg = (uint32_t)F.u(addr + 2, 2);
  uint32_t hsize = (uint32_t)F.u(addr + 8, 4);
  struct Block { uint64_t off, len; };
  std::vector<Block> blocks{{addr + 16, hsize}};
  uint32_t seen = 0;
  for (size_t b = 0; b < blocks.size() && seen < nmsg; ++b) {
    uint64_t p = blocks[b].off, end = blocks[b].off + blocks[b].len;
    if (!F.in(blocks[b].off, blocks[b].len)) return false;
    while (p + 8 <= end && seen < nmsg) {
      uint32_t type = (uint32_t)F.u(p, 2);
      uint32_t msz = (uint32_t)F.u(p + 2, 2);
      uint64_t d = p + 8;
      if (d + msz > end) return false;
      ++seen;
      if (type == 0x0001) {  // dataspace
        int ver = F.buf[d], rank = F.buf[d + 1];
        uint64_t q = (ver == 1) ? d + 8 : d + 4;
        ds.dims.clear();
        for (int i = 0; i < rank; ++i) ds.dims.push_back(F.u(q + (uint64_t)i * F.sl, F.sl));
      } else if (type == 0x0003) {  // datatype
        ds.fclass = F.buf[d] & 0x0f;
        ds.little = (F.buf[d + 1] & 1) == 0;
        ds.elsize = (int)F.u(d + 4, 4);
      } else if (type == 0x0008) {  // data layout
        int ver = F.buf[d];
        if (ver == 3) {
          ds.layout = F.buf[d + 1];
          if (ds.layout == 1) {
            ds.addr = F.u(d + 2, F.so);
            ds.size = F.u(d + 2 + F.so, F.sl);
          } else if (ds.layout == 0) {
            ds.size = F.u(d + 2, 2);
            ds.compact_off = d + 4;
          }
        } else if (ver == 1 || ver == 2) {
          int rank = F.buf[d + 1];
          ds.layout = F.buf[d + 2];
          if (ds.layout == 1) {
            ds.addr = F.u(d + 8, F.so);
            ds.size = 0;  // derived from the dataspace
          } else if (ds.layout == 0) {
            uint64_t q = d + 8 + (uint64_t)rank * 4;
            ds.size = F.u(q, 4);
            ds.compact_off = q + 4;
          }
        }
      } else if (type == 0x0010) {  // continuation
        blocks.push_back({F.u(d, F.so), F.u(d + F.so, F.sl)});
      } else if (type == 0x0011) {  // symbol table (group)
        if (btree) *btree = F.u(d, F.so);
        if (heap) *heap = F.u(d + F.so, F.so);
      }
      p = d + ((msz + 7u) & ~7u);
    }
  }
  return true;
}

// Walk a group's v1 B-tree, collecting name -> object header address.
bool walk_group(const H5File &F, uint64_t btree, uint64_t heap_data,
                std::map<std::string, uint64_t> &out, int depth = 0) {
  if (depth > 16 || !F.in(btree, 24) || std::memcmp(&F.buf[btree], "TREE", 4) != 0) return false;
  int level = F.buf[btree + 5];
  int used = (int)F.u(btree + 6, 2);
  uint64_t p = btree + 8 + 2 * (uint64_t)F.so;  // skip siblings
  p += F.sl;                                     // key 0
  for (int i = 0; i < used; ++i) {
    uint64_t child = F.u(p, F.so);
    p += F.so + F.sl;
    if (level > 0) {
      if (!walk_group(F, child, heap_data, out, depth + 1)) return false;
      continue;
    }
    if (!F.in(child, 8) || std::memcmp(&F.buf[child], "SNOD", 4) != 0) return false;
    int nsym = (int)F.u(child + 6, 2);
    uint64_t e = child + 8;
    for (int s = 0; s < nsym; ++s, e += 2 * F.so + 24) {
      if (!F.in(e, 2 * F.so + 24)) return false;
      uint64_t name_off = F.u(e, F.so), oh = F.u(e + F.so, F.so);
      uint64_t nm = heap_data + name_off;
      if (!F.in(nm, 1)) return false;
      std::string name((const char *)&F.buf[nm]);
      out[name] = oh;
    }
  }
  return true;
}

bool read_values(const H5File &F, const Dataset &ds, std::vector<double> &v) {
  uint64_t n = 1;
  for (auto d : ds.dims) n *= d;
  if (ds.fclass != 1 || !ds.little || (ds.elsize != 4 && ds.elsize != 8)) return false;
  uint64_t off = (ds.layout == 1) ? F.base + ds.addr : ds.compact_off;
  if (ds.layout != 0 && ds.layout != 1) return false;
  if (!F.in(off, n * (uint64_t)ds.elsize)) return false;
  v.resize(n);
  for (uint64_t i = 0; i < n; ++i) {
    if (ds.elsize == 8) {
      double x;
      std::memcpy(&x, &F.buf[off + 8 * i], 8);
      v[i] = x;
    } else {
      float x;
      std::memcpy(&x, &F.buf[off + 4 * i], 4);
      v[i] = (double)x;
    }
  }
  return true;
}

}  // namespace

extern "C" int hipft_h5_read(const char *path, int *ndim, int64_t dims[3], double *data, double *s1,
                             double *s2, double *s3) {
  if (!path || !ndim || !dims) return HIPFT_EINVAL;
  H5File F;
  if (!F.load(path)) return HIPFT_EIO;
  static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  uint64_t sb = 0;
  while (sb + 8 <= F.buf.size() && std::memcmp(&F.buf[sb], sig, 8) != 0) {
    sb = sb ? sb * 2 : 512;
    if (sb > F.buf.size()) return HIPFT_EIO;
  }
  if (!F.in(sb, 96)) return HIPFT_EIO;
  int ver = F.buf[sb + 8];
  if (ver > 1) return HIPFT_EIO;  // only superblock v0/v1 (libver "earliest")
  F.so = F.buf[sb + 13];
  F.sl = F.buf[sb + 14];
  if (F.so != 8 || F.sl != 8) return HIPFT_EIO;
  uint64_t p = sb + 24 + (ver == 1 ? 4 : 0);
  F.base = F.u(p, 8);
  uint64_t root_entry = p + 4 * 8;
  uint64_t root_oh = F.u(root_entry + 8, 8);
  uint64_t btree = 0, heap = 0;
  if (F.u(root_entry + 16, 4) == 1) {
    btree = F.u(root_entry + 24, 8);
    heap = F.u(root_entry + 32, 8);
  } else {
    Dataset dummy;
    if (!parse_object(F, F.base + root_oh, dummy, &btree, &heap)) return HIPFT_EIO;
  }
  if (!F.in(F.base + heap, 32) || std::memcmp(&F.buf[F.base + heap], "HEAP", 4) != 0) return HIPFT_EIO;
  uint64_t heap_data = F.base + F.u(F.base + heap + 24, 8);
  std::map<std::string, uint64_t> objs;
  if (!walk_group(F, F.base + btree, heap_data, objs)) return HIPFT_EIO;
  auto it = objs.find("Data");
  if (it == objs.end()) return HIPFT_EIO;
  Dataset D;
  if (!parse_object(F, F.base + it->second, D, nullptr, nullptr)) return HIPFT_EIO;
  int nd = (int)D.dims.size();
  if (nd < 1 || nd > 3) return HIPFT_EIO;
  *ndim = nd;
  for (int i = 0; i < 3; ++i) dims[i] = 1;
  for (int i = 0; i < nd; ++i) dims[i] = (int64_t)D.dims[nd - 1 - i];  // Fortran order
  if (!data && !s1 && !s2 && !s3) return HIPFT_OK;
  if (data) {
    std::vector<double> v;
    if (!read_values(F, D, v)) return HIPFT_EIO;
    std::memcpy(data, v.data(), v.size() * sizeof(double));
  }
  double *scales[3] = {s1, s2, s3};
  const char *names[3] = {"dim1", "dim2", "dim3"};
  for (int i = 0; i < nd; ++i) {
    if (!scales[i]) continue;
    auto s = objs.find(names[i]);
    if (s == objs.end()) return HIPFT_EIO;
    Dataset S;
    if (!parse_object(F, F.base + s->second, S, nullptr, nullptr)) return HIPFT_EIO;
    std::vector<double> v;
    if (!read_values(F, S, v) || (int64_t)v.size() != dims[i]) return HIPFT_EIO;
    std::memcpy(scales[i], v.data(), v.size() * sizeof(double));
  }
  return HIPFT_OK;
}
