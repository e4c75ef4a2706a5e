// h5lite.hh -- one N-dimensional floating-point dataset in an HDF5 file, without libhdf5.
//
// The reference stores a field as the dataset "/stochastic" of "<name>.stoch.h5"
// (io.hh:170-270: H5Fcreate with default properties, H5Dcreate of an H5T_IEEE_F64LE
// dataset whose dimensions are the cells in reverse order, contiguous storage), read back
// by io.hh:55-150.  This image has no HDF5 library, so the file is written and read here
// from the structures of the HDF5 file format specification (version 0 superblock, a root
// group with a symbol table: v1 B-tree of group nodes, symbol table node and local heap,
// version 1 object headers, dataspace / datatype / contiguous layout messages), which is
// what the library's default properties produce for such a file.
//
// Writer: superblock v0 (offsets and lengths of 8 bytes, group leaf / internal node K 4 /
// 16), root group object header, root local heap, root B-tree node, one symbol table node,
// the dataset object header and the raw data, little-endian, all at 8-byte aligned offsets.
// Reader: superblock v0 or v1, symbol-table groups (B-tree levels walked), version 1 object
// headers with continuation messages, dataspace v1/v2, IEEE float datatypes of 4 or 8
// bytes (little-endian), contiguous layout v3; anything else is reported as unsupported.
#pragma once

#include <cstdint>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace parafields_b200 {
namespace h5lite {

constexpr uint64_t kUndef = ~0ull;

namespace detail {

struct Buf {
  std::vector<unsigned char> b;
  size_t at(size_t pos) {
    if (b.size() < pos) b.resize(pos, 0);
    return pos;
  }
  void put(size_t pos, uint64_t v, int n) {
    if (b.size() < pos + n) b.resize(pos + n, 0);
    for (int i = 0; i < n; i++) b[pos + i] = (unsigned char)(v >> (8 * i));
  }
  void bytes(size_t pos, const void* p, size_t n) {
    if (b.size() < pos + n) b.resize(pos + n, 0);
    std::memcpy(b.data() + pos, p, n);
  }
};

inline size_t align8(size_t x) { return (x + 7) & ~size_t(7); }

// version 1 object header: 16-byte prefix, then messages (type, size, flags) padded to 8
// bytes; the remainder up to `min_data` bytes is one NIL message
struct Msg {
  uint16_t type;
  std::vector<unsigned char> data;
};
inline size_t object_header(Buf& f, size_t pos, std::vector<Msg> msgs, size_t min_data = 256) {
  size_t data = 0;
  for (auto& m : msgs) {
    m.data.resize(align8(m.data.size()), 0);
    data += 8 + m.data.size();
  }
  if (data + 8 <= min_data) {
    msgs.push_back({0, std::vector<unsigned char>(min_data - data - 8, 0)});
    data = min_data;
  }
  f.put(pos, 1, 1);                // version
  f.put(pos + 2, msgs.size(), 2);  // number of messages
  f.put(pos + 4, 1, 4);            // reference count
  f.put(pos + 8, data, 4);         // header data size
  size_t p = pos + 16;
  for (const auto& m : msgs) {
    f.put(p, m.type, 2);
    f.put(p + 2, m.data.size(), 2);
    f.put(p + 4, 0, 1);
    if (!m.data.empty()) f.bytes(p + 8, m.data.data(), m.data.size());
    p += 8 + m.data.size();
  }
  return p;
}

inline void le(std::vector<unsigned char>& v, uint64_t x, int n) {
  for (int i = 0; i < n; i++) v.push_back((unsigned char)(x >> (8 * i)));
}

}  // namespace detail

// Writes `data` (prod(dims) values, last dimension fastest, i.e. HDF5's C order) as the
// dataset `name` of a new file `path`, stored as IEEE little-endian floats of
// `file_bytes` (8: H5T_IEEE_F64LE, 4: H5T_IEEE_F32LE) bytes.
template <typename T>
void write(const std::string& path, const std::string& name, const std::vector<uint64_t>& dims, const T* data,
           int file_bytes = 8) {
  using namespace detail;
  if (dims.empty() || dims.size() > 32) throw std::runtime_error{"h5lite: rank must be 1..32"};
  if (file_bytes != 4 && file_bytes != 8) throw std::runtime_error{"h5lite: element size must be 4 or 8"};
  if (name.empty() || name.find('/') != std::string::npos) throw std::runtime_error{"h5lite: bad dataset name"};
  uint64_t count = 1;
  for (uint64_t d : dims) count *= d;
  Buf f;
  const size_t SB = 0, ROOT_OH = 96;
  // root group: symbol table message (B-tree and heap addresses filled in below)
  const size_t HEAP = align8(ROOT_OH + 16 + 256);
  const size_t HEAP_DATA = HEAP + 32;
  const size_t name_off = 8;
  const size_t heap_size = align8(name_off + name.size() + 1);
  const size_t BTREE = align8(HEAP_DATA + heap_size);
  const int leaf_k = 4, internal_k = 16;
  const size_t btree_size = 24 + 2 * internal_k * 8 + (2 * internal_k + 1) * 8;
  const size_t SNOD = align8(BTREE + btree_size);
  const size_t snod_size = 8 + 2 * leaf_k * 40;
  const size_t DSET_OH = align8(SNOD + snod_size);
  // dataset object header
  std::vector<Msg> dm;
  {
    Msg space{0x0001, {}};
    space.data = {1, (unsigned char)dims.size(), 0, 0, 0, 0, 0, 0};
    for (uint64_t d : dims) le(space.data, d, 8);
    Msg type{0x0003, {}};
    const bool f8 = file_bytes == 8;
    type.data = {0x11, 0x20, (unsigned char)(f8 ? 63 : 31), 0};  // v1 float, LE, implied msb, sign bit
    le(type.data, (uint64_t)file_bytes, 4);
    le(type.data, 0, 2);                           // bit offset
    le(type.data, (uint64_t)(f8 ? 64 : 32), 2);    // precision
    type.data.push_back((unsigned char)(f8 ? 52 : 23));  // exponent location
    type.data.push_back((unsigned char)(f8 ? 11 : 8));   // exponent size
    type.data.push_back(0);                              // mantissa location
    type.data.push_back((unsigned char)(f8 ? 52 : 23));  // mantissa size
    le(type.data, (uint64_t)(f8 ? 1023 : 127), 4);        // exponent bias
    Msg layout{0x0008, {3, 1}};
    dm = {space, type, layout};
  }
  // the layout message needs the data address: size the header first
  size_t dset_end = 0;
  {
    Buf tmp;
    std::vector<Msg> probe = dm;
    probe[2].data.resize(2 + 16, 0);
    dset_end = object_header(tmp, 0, probe) + DSET_OH;
  }
  const size_t DATA = align8(dset_end);
  const uint64_t data_bytes = count * (uint64_t)file_bytes;
  le(dm[2].data, DATA, 8);
  le(dm[2].data, data_bytes, 8);
  object_header(f, DSET_OH, dm);
  // root object header
  {
    Msg st{0x0011, {}};
    le(st.data, BTREE, 8);
    le(st.data, HEAP, 8);
    object_header(f, ROOT_OH, {st});
  }
  // local heap: "" at 0, the dataset name at 8, no free block (free-list head 1)
  f.bytes(HEAP, "HEAP", 4);
  f.put(HEAP + 4, 0, 1);
  f.put(HEAP + 8, heap_size, 8);
  f.put(HEAP + 16, 1, 8);
  f.put(HEAP + 24, HEAP_DATA, 8);
  f.at(HEAP_DATA + heap_size);
  f.bytes(HEAP_DATA + name_off, name.c_str(), name.size() + 1);
  // B-tree group node (level 0, one child: the symbol table node)
  f.bytes(BTREE, "TREE", 4);
  f.put(BTREE + 4, 0, 1);  // node type: group
  f.put(BTREE + 5, 0, 1);  // level
  f.put(BTREE + 6, 1, 2);  // entries used
  f.put(BTREE + 8, kUndef, 8);
  f.put(BTREE + 16, kUndef, 8);
  f.put(BTREE + 24, 0, 8);         // key 0: heap offset of ""
  f.put(BTREE + 32, SNOD, 8);      // child 0
  f.put(BTREE + 40, name_off, 8);  // key 1: largest name in child 0
  f.at(BTREE + btree_size);
  // symbol table node with one entry
  f.bytes(SNOD, "SNOD", 4);
  f.put(SNOD + 4, 1, 1);
  f.put(SNOD + 6, 1, 2);
  f.put(SNOD + 8, name_off, 8);
  f.put(SNOD + 16, DSET_OH, 8);
  f.put(SNOD + 24, 0, 4);  // cache type: nothing cached
  f.at(SNOD + snod_size);
  // raw data
  const size_t eof = DATA + data_bytes;
  // superblock v0
  static const unsigned char sig[8] = {0x89, 'H', 'D', 'F', 0x0d, 0x0a, 0x1a, 0x0a};
  f.bytes(SB, sig, 8);
  f.put(SB + 8, 0, 1);    // superblock version
  f.put(SB + 9, 0, 1);    // free-space version
  f.put(SB + 10, 0, 1);   // root group symbol table entry version
  f.put(SB + 12, 0, 1);   // shared header message format version
  f.put(SB + 13, 8, 1);   // size of offsets
  f.put(SB + 14, 8, 1);   // size of lengths
  f.put(SB + 16, leaf_k, 2);
  f.put(SB + 18, internal_k, 2);
  f.put(SB + 20, 0, 4);   // consistency flags
  f.put(SB + 24, 0, 8);   // base address
  f.put(SB + 32, kUndef, 8);  // free-space info
  f.put(SB + 40, eof, 8);     // end of file
  f.put(SB + 48, kUndef, 8);  // driver information block
  f.put(SB + 56, 0, 8);       // root entry: link name offset
  f.put(SB + 64, ROOT_OH, 8);
  f.put(SB + 72, 1, 4);       // cache type 1: B-tree and heap addresses in the scratch pad
  f.put(SB + 80, BTREE, 8);
  f.put(SB + 88, HEAP, 8);
  std::ofstream out(path, std::ios::binary | std::ios::trunc);
  if (!out) throw std::runtime_error{"h5lite: cannot create " + path};
  f.at(DATA);
  out.write((const char*)f.b.data(), (std::streamsize)f.b.size());
  std::vector<unsigned char> chunk;
  const uint64_t per = 1u << 16;
  for (uint64_t i = 0; i < count; i += per) {
    const uint64_t n = count - i < per ? count - i : per;
    chunk.resize((size_t)(n * file_bytes));
    for (uint64_t k = 0; k < n; k++) {
      if (file_bytes == 8) {
        const double v = (double)data[i + k];
        std::memcpy(&chunk[(size_t)k * 8], &v, 8);
      } else {
        const float v = (float)data[i + k];
        std::memcpy(&chunk[(size_t)k * 4], &v, 4);
      }
    }
    out.write((const char*)chunk.data(), (std::streamsize)chunk.size());
  }
  if (!out) throw std::runtime_error{"h5lite: write to " + path + " failed"};
}

namespace detail {

struct Reader {
  std::ifstream in;
  std::string path;
  uint64_t base = 0;
  std::vector<unsigned char> get(uint64_t addr, size_t n) {
    std::vector<unsigned char> v(n);
    in.clear();
    in.seekg((std::streamoff)(base + addr));
    in.read((char*)v.data(), (std::streamsize)n);
    if (!in) throw std::runtime_error{"h5lite: " + path + " is truncated or not an HDF5 file"};
    return v;
  }
  static uint64_t u(const std::vector<unsigned char>& v, size_t pos, int n) {
    if (pos + n > v.size()) throw std::runtime_error{"h5lite: structure overruns its block"};
    uint64_t x = 0;
    for (int i = 0; i < n; i++) x |= (uint64_t)v[pos + i] << (8 * i);
    return x;
  }
  // messages of a version 1 object header (following continuation messages)
  std::vector<std::pair<uint16_t, std::vector<unsigned char>>> messages(uint64_t addr) {
    const auto pre = get(addr, 16);
    if (pre[0] != 1) throw std::runtime_error{"h5lite: only version 1 object headers are supported"};
    std::vector<std::pair<uint16_t, std::vector<unsigned char>>> out;
    std::vector<std::pair<uint64_t, uint64_t>> chunks = {{addr + 16, u(pre, 8, 4)}};
    for (size_t c = 0; c < chunks.size() && c < 64; c++) {
      const auto blk = get(chunks[c].first, (size_t)chunks[c].second);
      size_t p = 0;
      while (p + 8 <= blk.size()) {
        const uint16_t type = (uint16_t)u(blk, p, 2);
        const size_t size = (size_t)u(blk, p + 2, 2);
        if (p + 8 + size > blk.size()) throw std::runtime_error{"h5lite: malformed object header"};
        std::vector<unsigned char> data(blk.begin() + p + 8, blk.begin() + p + 8 + size);
        if (type == 0x0010) chunks.push_back({u(data, 0, 8), u(data, 8, 8)});
        out.push_back({type, std::move(data)});
        p += 8 + size;
      }
    }
    return out;
  }
  // object header address of `name` in the symbol-table group of B-tree `btree`
  uint64_t lookup(uint64_t btree, uint64_t heap_data, const std::string& name, int depth = 0) {
    if (depth > 16) throw std::runtime_error{"h5lite: B-tree too deep"};
    const auto hdr = get(btree, 24);
    if (std::memcmp(hdr.data(), "TREE", 4) != 0 || hdr[4] != 0) throw std::runtime_error{"h5lite: bad group B-tree"};
    const int level = hdr[5];
    const int used = (int)u(hdr, 6, 2);
    const auto kv = get(btree + 24, (size_t)(16 * used + 8));
    for (int i = 0; i < used; i++) {
      const uint64_t child = u(kv, 8 + 16 * i, 8);
      if (level > 0) {
        const uint64_t r = lookup(child, heap_data, name, depth + 1);
        if (r != kUndef) return r;
        continue;
      }
      const auto sh = get(child, 8);
      if (std::memcmp(sh.data(), "SNOD", 4) != 0) throw std::runtime_error{"h5lite: bad symbol table node"};
      const int n = (int)u(sh, 6, 2);
      const auto ents = get(child + 8, (size_t)(40 * n));
      for (int e = 0; e < n; e++) {
        const auto nm = get(heap_data + u(ents, 40 * e, 8), name.size() + 1);
        if (std::memcmp(nm.data(), name.c_str(), name.size() + 1) == 0) return u(ents, 40 * e + 8, 8);
      }
    }
    return kUndef;
  }
};

}  // namespace detail

// Reads dataset `name` of `path` (dimensions into *dims, slowest first) as doubles.
inline std::vector<double> read(const std::string& path, const std::string& name, std::vector<uint64_t>* dims) {
  using detail::Reader;
  Reader r;
  r.path = path;
  r.in.open(path, std::ios::binary);
  if (!r.in) throw std::runtime_error{"h5lite: cannot open " + path};
  const auto sb = r.get(0, 8);
  static const unsigned char sig[8] = {0x89, 'H', 'D', 'F', 0x0d, 0x0a, 0x1a, 0x0a};
  if (std::memcmp(sb.data(), sig, 8) != 0) throw std::runtime_error{"h5lite: " + path + " is not an HDF5 file"};
  const auto s = r.get(0, 128);
  const int ver = s[8];
  if (ver > 1) throw std::runtime_error{"h5lite: superblock version " + std::to_string(ver) + " is not supported"};
  if (s[13] != 8 || s[14] != 8) throw std::runtime_error{"h5lite: only 8-byte offsets and lengths are supported"};
  const size_t a = ver == 0 ? 24 : 28;  // v1 adds the indexed storage K and a reserved word
  r.base = Reader::u(s, a, 8);
  const uint64_t root_oh = Reader::u(s, a + 32 + 8, 8);
  uint64_t btree = kUndef, heap = kUndef;
  for (const auto& m : r.messages(root_oh))
    if (m.first == 0x0011) {
      btree = Reader::u(m.second, 0, 8);
      heap = Reader::u(m.second, 8, 8);
    }
  if (btree == kUndef) throw std::runtime_error{"h5lite: the root group has no symbol table"};
  const auto hh = r.get(heap, 32);
  if (std::memcmp(hh.data(), "HEAP", 4) != 0) throw std::runtime_error{"h5lite: bad local heap"};
  const uint64_t oh = r.lookup(btree, Reader::u(hh, 24, 8), name);
  if (oh == kUndef) throw std::runtime_error{"h5lite: dataset /" + name + " not found in " + path};
  std::vector<uint64_t> dd;
  int esize = 0;
  uint64_t addr = kUndef, bytes = 0;
  for (const auto& m : r.messages(oh)) {
    const auto& d = m.second;
    if (m.first == 0x0001) {
      const int rank = d[1];
      const size_t off = d[0] == 1 ? 8 : 4;
      dd.clear();
      for (int i = 0; i < rank; i++) dd.push_back(Reader::u(d, off + 8 * i, 8));
    } else if (m.first == 0x0003) {
      if ((d[0] & 0x0f) != 1) throw std::runtime_error{"h5lite: dataset is not floating point"};
      if (d[1] & 1) throw std::runtime_error{"h5lite: big-endian data is not supported"};
      esize = (int)Reader::u(d, 4, 4);
    } else if (m.first == 0x0008) {
      if (d[0] != 3 || d[1] != 1) throw std::runtime_error{"h5lite: only contiguous layout (v3) is supported"};
      addr = Reader::u(d, 2, 8);
      bytes = Reader::u(d, 10, 8);
    }
  }
  if (esize != 4 && esize != 8) throw std::runtime_error{"h5lite: element size must be 4 or 8"};
  uint64_t count = 1;
  for (uint64_t x : dd) count *= x;
  if (addr == kUndef || bytes != count * (uint64_t)esize) throw std::runtime_error{"h5lite: inconsistent dataset storage"};
  std::vector<double> out((size_t)count);
  const uint64_t per = 1u << 16;
  for (uint64_t i = 0; i < count; i += per) {
    const uint64_t n = count - i < per ? count - i : per;
    const auto raw = r.get(addr + i * esize, (size_t)(n * esize));
    for (uint64_t k = 0; k < n; k++) {
      if (esize == 8) {
        std::memcpy(&out[(size_t)(i + k)], &raw[(size_t)k * 8], 8);
      } else {
        float v;
        std::memcpy(&v, &raw[(size_t)k * 4], 4);
        out[(size_t)(i + k)] = v;
      }
    }
  }
  if (dims) *dims = dd;
  return out;
}

}  // namespace h5lite
}  // namespace parafields_b200
