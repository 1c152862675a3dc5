// h5mini.cpp -- see h5mini.h.  Structure names and field orders follow the
// HDF5 file format specification: superblock, object header (v1, v2),
// header messages (dataspace 0x1, link info 0x2, datatype 0x3, fill value
// 0x5, link 0x6, data layout 0x8, filter pipeline 0xB, continuation 0x10,
// symbol table 0x11), v1 B-tree ("TREE"), symbol table node ("SNOD") and
// local heap ("HEAP").
#include "h5mini.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

namespace h5m {

namespace {

constexpr uint64_t kUndef = ~0ull;
const uint8_t kSig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

// ---------------------------------------------------------------------------
// read side
// ---------------------------------------------------------------------------
struct Msg {
  unsigned type;
  uint64_t off; // absolute offset of the message data
  uint64_t size;
};

struct Entry {
  std::string name;
  uint64_t ohdr;
};

struct SymTab {
  uint64_t btree = kUndef, heap = kUndef;
  uint64_t msg_off = 0; // absolute offset of the message data (for relinking)
};

class Reader {
public:
  ~Reader()
  {
    if (map_ && map_ != MAP_FAILED)
      munmap(const_cast<uint8_t *>(map_), len_);
    if (fd_ >= 0)
      close(fd_);
  }

  bool open(const std::string &path, std::string &err)
  {
    fd_ = ::open(path.c_str(), O_RDONLY);
    if (fd_ < 0)
      return fail(err, "cannot open " + path);
    struct stat st;
    if (fstat(fd_, &st) || st.st_size < 48)
      return fail(err, path + " is not an HDF5 file (too short)");
    len_ = (uint64_t)st.st_size;
    void *m = mmap(nullptr, len_, PROT_READ, MAP_PRIVATE, fd_, 0);
    if (m == MAP_FAILED)
      return fail(err, "cannot map " + path);
    map_ = static_cast<const uint8_t *>(m);
    // the superblock sits at 0, 512, 1024, ... (user block before it)
    for (uint64_t at = 0u; at + 8u <= len_; at = at ? at * 2u : 512u) {
      if (!std::memcmp(map_ + at, kSig, 8)) {
        sb_ = at;
        break;
      }
      if (at > (1ull << 40))
        break;
    }
    if (sb_ == kUndef)
      return fail(err, path + ": no HDF5 signature");
    return parse_superblock(err);
  }

  uint64_t u(uint64_t off, unsigned n) const
  { // little-endian unsigned of n bytes; out-of-range reads give kUndef
    if (off > len_ || n > len_ - off || n > 8u)
      return kUndef;
    uint64_t v = 0u;
    for (unsigned i = 0u; i < n; ++i)
      v |= (uint64_t)map_[off + i] << (8u * i);
    return v;
  }
  uint64_t addr(uint64_t off) const
  {
    const uint64_t v = u(off, so_);
    if (so_ < 8u && v == ((1ull << (8u * so_)) - 1u))
      return kUndef;
    return (v == kUndef) ? kUndef : v + base_;
  }
  bool in(uint64_t off, uint64_t n) const { return off <= len_ && n <= len_ - off; }
  const uint8_t *at(uint64_t off) const { return map_ + off; }

  unsigned so() const { return so_; }
  unsigned sl() const { return sl_; }
  unsigned version() const { return ver_; }
  uint64_t root() const { return root_; }
  uint64_t sb() const { return sb_; }
  uint64_t size() const { return len_; }

  bool messages(uint64_t oh, std::vector<Msg> &out, std::string &err) const
  {
    out.clear();
    if (!in(oh, 16))
      return fail(err, "object header out of range");
    if (!std::memcmp(at(oh), "OHDR", 4))
      return messages_v2(oh, out, err);
    if (map_[oh] != 1u)
      return fail(err, "unknown object header version");
    const unsigned nmsg = (unsigned)u(oh + 2u, 2);
    const uint64_t hsize = u(oh + 8u, 4);
    std::vector<std::pair<uint64_t, uint64_t>> blocks{{oh + 16u, hsize}};
    unsigned seen = 0u;
    for (size_t b = 0u; b < blocks.size() && seen < nmsg; ++b) {
      uint64_t p = blocks[b].first;
      const uint64_t end = p + blocks[b].second;
      if (!in(blocks[b].first, blocks[b].second))
        return fail(err, "object header block out of range");
      while (p + 8u <= end && seen < nmsg) {
        const unsigned type = (unsigned)u(p, 2);
        const uint64_t size = u(p + 2u, 2);
        if (p + 8u + size > end)
          return fail(err, "object header message overruns its block");
        ++seen;
        if (type == 0x10u)
          blocks.push_back({addr(p + 8u), u(p + 8u + so_, sl_)});
        else
          out.push_back({type, p + 8u, size});
        p += 8u + size;
      }
      if (blocks.size() > 1024u)
        return fail(err, "too many header continuation blocks");
    }
    return true;
  }

  bool symtab(const std::vector<Msg> &ms, SymTab &st) const
  {
    for (const Msg &m : ms)
      if (m.type == 0x11u) {
        st.btree = addr(m.off);
        st.heap = addr(m.off + so_);
        st.msg_off = m.off;
        return true;
      }
    return false;
  }

  // all (name, object header) entries of a group
  bool entries(uint64_t oh, std::vector<Entry> &out, std::string &err) const
  {
    out.clear();
    std::vector<Msg> ms;
    if (!messages(oh, ms, err))
      return false;
    SymTab st;
    if (symtab(ms, st)) {
      uint64_t heap_data = 0u, heap_size = 0u;
      if (!heap(st.heap, heap_data, heap_size, err))
        return false;
      return btree_entries(st.btree, heap_data, heap_size, out, err, 0);
    }
    bool any = false;
    for (const Msg &m : ms) {
      if (m.type == 0x02u) { // link info: dense storage if the fractal heap exists
        const unsigned fl = map_[m.off + 1u];
        const uint64_t fh = addr(m.off + 2u + ((fl & 1u) ? 8u : 0u));
        if (fh != kUndef)
          return fail(err, "groups with dense (fractal heap) link storage are not supported");
      }
      if (m.type != 0x06u)
        continue;
      any = true;
      Entry e;
      if (!link(m, e, err))
        return false;
      if (e.ohdr != kUndef)
        out.push_back(e);
    }
    (void)any;
    return true;
  }

  bool lookup(const std::string &path, uint64_t &oh, std::string &err) const
  {
    oh = root_;
    size_t p = 0u;
    while (p < path.size()) {
      size_t q = path.find('/', p);
      if (q == std::string::npos)
        q = path.size();
      const std::string part = path.substr(p, q - p);
      p = q + 1u;
      if (part.empty() || part == ".")
        continue;
      std::vector<Entry> es;
      if (!entries(oh, es, err))
        return false;
      bool found = false;
      for (const Entry &e : es)
        if (e.name == part) {
          oh = e.ohdr;
          found = true;
          break;
        }
      if (!found)
        return fail(err, "no object named " + part);
    }
    return true;
  }

  bool dataset(uint64_t oh, Array &a, uint64_t *data_addr, std::string &err) const
  {
    std::vector<Msg> ms;
    if (!messages(oh, ms, err))
      return false;
    const Msg *sp = nullptr, *ty = nullptr, *ly = nullptr;
    for (const Msg &m : ms) {
      if (m.type == 0x01u)
        sp = &m;
      else if (m.type == 0x03u)
        ty = &m;
      else if (m.type == 0x08u)
        ly = &m;
      else if (m.type == 0x0Bu)
        return fail(err, "filtered (compressed) datasets are not supported");
    }
    if (!sp || !ty || !ly)
      return fail(err, "not a dataset");
    if (!dataspace(*sp, a.dims, err) || !datatype(*ty, a, err))
      return false;
    // the byte count must not wrap: every extent defined, and the product of
    // the extents and the element size no larger than the file (a dataset
    // stored in the file cannot be longer than the file)
    uint64_t need = a.size;
    for (const uint64_t d : a.dims) {
      if (d == kUndef)
        return fail(err, "dataset with an undefined extent");
      if (d && need > len_ / d)
        return fail(err, "dataset larger than the file");
      need *= d;
    }
    uint64_t daddr = kUndef, dsize = 0u;
    const uint8_t *compact = nullptr;
    if (!layout(*ly, (unsigned)a.dims.size(), daddr, dsize, compact, err))
      return false;
    a.raw.assign(need, 0u);
    if (compact) {
      if (dsize < need)
        return fail(err, "compact dataset shorter than its dataspace");
      std::memcpy(a.raw.data(), compact, need);
    }
    else if (daddr != kUndef) {
      if (!in(daddr, need))
        return fail(err, "dataset data out of range");
      std::memcpy(a.raw.data(), at(daddr), need);
    } // unallocated: zeros (the default fill value)
    if (data_addr)
      *data_addr = compact ? kUndef : daddr;
    return true;
  }

private:
  static bool fail(std::string &err, const std::string &m)
  {
    err = m;
    return false;
  }

  bool parse_superblock(std::string &err)
  {
    const uint64_t s = sb_;
    ver_ = map_[s + 8u];
    if (ver_ <= 1u) {
      so_ = map_[s + 13u];
      sl_ = map_[s + 14u];
      if (so_ < 2u || so_ > 8u || sl_ < 2u || sl_ > 8u)
        return fail(err, "bad sizes in superblock");
      uint64_t p = s + 24u + (ver_ == 1u ? 4u : 0u);
      base_ = u(p, so_);
      p += 4u * so_;                     // base, free space, end of file, driver
      root_ = u(p + so_, so_) + base_;   // root symbol table entry: name offset, header
    }
    else if (ver_ == 2u || ver_ == 3u) {
      so_ = map_[s + 9u];
      sl_ = map_[s + 10u];
      if (so_ < 2u || so_ > 8u || sl_ < 2u || sl_ > 8u)
        return fail(err, "bad sizes in superblock");
      const uint64_t p = s + 12u;
      base_ = u(p, so_);
      root_ = u(p + 3u * so_, so_) + base_; // base, extension, end of file, root header
    }
    else
      return fail(err, "unsupported superblock version");
    if (base_ == kUndef || !in(root_, 8))
      return fail(err, "bad root group address");
    return true;
  }

  bool messages_v2(uint64_t oh, std::vector<Msg> &out, std::string &err) const
  {
    const unsigned flags = map_[oh + 5u];
    uint64_t p = oh + 6u;
    if (flags & 0x20u)
      p += 16u;
    if (flags & 0x10u)
      p += 4u;
    const unsigned nb = 1u << (flags & 3u);
    const uint64_t size = u(p, nb);
    p += nb;
    std::vector<std::pair<uint64_t, uint64_t>> blocks{{p, size}};
    const unsigned mh = 4u + ((flags & 0x04u) ? 2u : 0u);
    for (size_t b = 0u; b < blocks.size(); ++b) {
      uint64_t q = blocks[b].first;
      const uint64_t end = q + blocks[b].second;
      if (!in(blocks[b].first, blocks[b].second))
        return fail(err, "object header block out of range");
      while (q + mh <= end) {
        const unsigned type = map_[q];
        const uint64_t msz = u(q + 1u, 2);
        const uint64_t d = q + mh;
        if (d + msz > end)
          return fail(err, "object header message overruns its block");
        if (type == 0x10u) {
          const uint64_t ca = addr(d), cl = u(d + so_, sl_);
          if (ca == kUndef || !in(ca, cl) || cl < 8u || std::memcmp(at(ca), "OCHK", 4))
            return fail(err, "bad object header continuation");
          blocks.push_back({ca + 4u, cl - 8u}); // signature, messages, checksum
        }
        else if (type != 0u)
          out.push_back({type, d, msz});
        q = d + msz;
      }
      if (blocks.size() > 1024u)
        return fail(err, "too many header continuation blocks");
    }
    return true;
  }

  bool heap(uint64_t h, uint64_t &data, uint64_t &size, std::string &err) const
  {
    if (!in(h, 8u + 2u * sl_ + so_) || std::memcmp(at(h), "HEAP", 4))
      return fail(err, "bad local heap");
    size = u(h + 8u, sl_);
    data = addr(h + 8u + 2u * sl_);
    if (!in(data, size))
      return fail(err, "local heap data out of range");
    return true;
  }

  bool heap_name(uint64_t data, uint64_t size, uint64_t off, std::string &name, std::string &err) const
  {
    if (off >= size)
      return fail(err, "name offset outside the local heap");
    const char *c = reinterpret_cast<const char *>(at(data + off));
    const size_t n = strnlen(c, size - off);
    name.assign(c, n);
    return true;
  }

  bool btree_entries(uint64_t node, uint64_t hd, uint64_t hs, std::vector<Entry> &out, std::string &err,
                     unsigned depth) const
  {
    if (node == kUndef)
      return true;
    if (depth > 64u || !in(node, 8u + 2u * so_) || std::memcmp(at(node), "TREE", 4) || map_[node + 4u] != 0u)
      return fail(err, "bad group B-tree node");
    const unsigned level = map_[node + 5u];
    const unsigned used = (unsigned)u(node + 6u, 2);
    uint64_t p = node + 8u + 2u * so_;
    for (unsigned i = 0u; i < used; ++i) {
      const uint64_t child = addr(p + sl_); // key, child, key, child, ..., key
      p += sl_ + so_;
      if (level) {
        if (!btree_entries(child, hd, hs, out, err, depth + 1u))
          return false;
        continue;
      }
      if (!in(child, 8u) || std::memcmp(at(child), "SNOD", 4))
        return fail(err, "bad symbol table node");
      const unsigned ns = (unsigned)u(child + 6u, 2);
      const uint64_t esz = 2u * so_ + 24u;
      if (!in(child + 8u, ns * esz))
        return fail(err, "symbol table node out of range");
      for (unsigned k = 0u; k < ns; ++k) {
        const uint64_t e = child + 8u + k * esz;
        Entry en;
        if (!heap_name(hd, hs, u(e, so_), en.name, err))
          return false;
        en.ohdr = addr(e + so_);
        out.push_back(en);
      }
    }
    return true;
  }

  bool link(const Msg &m, Entry &e, std::string &err) const
  {
    uint64_t p = m.off;
    if (map_[p] != 1u)
      return fail(err, "unknown link message version");
    const unsigned fl = map_[p + 1u];
    p += 2u;
    unsigned type = 0u;
    if (fl & 0x08u)
      type = map_[p++];
    if (fl & 0x04u)
      p += 8u;
    if (fl & 0x10u)
      p += 1u;
    const unsigned nb = 1u << (fl & 3u);
    const uint64_t nlen = u(p, nb);
    p += nb;
    if (!in(p, nlen))
      return fail(err, "link name out of range");
    e.name.assign(reinterpret_cast<const char *>(at(p)), nlen);
    p += nlen;
    e.ohdr = (type == 0u) ? addr(p) : kUndef; // soft and external links are skipped
    return true;
  }

  bool dataspace(const Msg &m, std::vector<uint64_t> &dims, std::string &err) const
  {
    const unsigned ver = map_[m.off], rank = map_[m.off + 1u];
    uint64_t p;
    if (ver == 1u)
      p = m.off + 8u;
    else if (ver == 2u) {
      if (map_[m.off + 3u] == 2u)
        return fail(err, "null dataspace");
      p = m.off + 4u;
    }
    else
      return fail(err, "unknown dataspace version");
    dims.clear();
    for (unsigned i = 0u; i < rank; ++i)
      dims.push_back(u(p + (uint64_t)i * sl_, sl_));
    return true;
  }

  bool datatype(const Msg &m, Array &a, std::string &err) const
  {
    const unsigned cls = map_[m.off] & 0x0fu;
    const unsigned b0 = map_[m.off + 1u];
    a.size = (unsigned)u(m.off + 4u, 4);
    if (cls == 0u) {
      if (b0 & 1u)
        return fail(err, "big-endian integers are not supported");
      if (a.size != 1u && a.size != 2u && a.size != 4u && a.size != 8u)
        return fail(err, "unsupported integer size");
      a.cls = 0;
      a.is_signed = (b0 & 0x08u) != 0u;
      return true;
    }
    if (cls == 1u) {
      if (b0 & 0x41u)
        return fail(err, "big-endian or VAX floats are not supported");
      const unsigned es = map_[m.off + 8u + 5u], ms = map_[m.off + 8u + 7u];
      if (!((a.size == 8u && es == 11u && ms == 52u) || (a.size == 4u && es == 8u && ms == 23u)))
        return fail(err, "only IEEE binary32/binary64 floats are supported");
      a.cls = 1;
      return true;
    }
    return fail(err, "unsupported datatype class");
  }

  bool layout(const Msg &m, unsigned rank, uint64_t &daddr, uint64_t &dsize, const uint8_t *&compact,
              std::string &err) const
  {
    const unsigned ver = map_[m.off];
    compact = nullptr;
    if (ver == 3u || ver == 4u) {
      const unsigned cls = map_[m.off + 1u];
      if (cls == 0u) {
        dsize = u(m.off + 2u, 2);
        compact = at(m.off + 4u);
        return in(m.off + 4u, dsize) || fail(err, "compact data out of range");
      }
      if (cls == 1u) {
        daddr = addr(m.off + 2u);
        dsize = u(m.off + 2u + so_, sl_);
        return true;
      }
      return fail(err, "chunked and virtual datasets are not supported");
    }
    if (ver == 1u || ver == 2u) {
      const unsigned cls = map_[m.off + 2u];
      uint64_t p = m.off + 8u;
      if (cls == 1u) {
        daddr = addr(p);
        dsize = kUndef;
        return true;
      }
      if (cls == 0u) {
        p += 4u * (uint64_t)map_[m.off + 1u];
        dsize = u(p, 4);
        compact = at(p + 4u);
        (void)rank;
        return in(p + 4u, dsize) || fail(err, "compact data out of range");
      }
      return fail(err, "chunked datasets are not supported");
    }
    return fail(err, "unknown layout message version");
  }

  int fd_ = -1;
  const uint8_t *map_ = nullptr;
  uint64_t len_ = 0u, sb_ = kUndef, base_ = 0u, root_ = kUndef;
  unsigned so_ = 8u, sl_ = 8u, ver_ = 0u;
};

} // namespace

uint64_t Array::count() const
{
  uint64_t c = 1u;
  for (uint64_t d : dims)
    c *= d;
  return c;
}

bool Array::to_double(std::vector<double> &out) const
{
  const uint64_t n = count();
  out.resize(n);
  for (uint64_t i = 0u; i < n; ++i) {
    const uint8_t *p = raw.data() + i * size;
    if (cls == 1 && size == 8u)
      std::memcpy(&out[i], p, 8);
    else if (cls == 1 && size == 4u) {
      float f;
      std::memcpy(&f, p, 4);
      out[i] = f;
    }
    else {
      uint64_t v = 0u;
      std::memcpy(&v, p, size);
      if (is_signed && size < 8u && (v >> (8u * size - 1u)))
        v |= ~0ull << (8u * size);
      out[i] = is_signed ? (double)(int64_t)v : (double)v;
    }
  }
  return true;
}

bool Array::to_int(std::vector<int> &out) const
{
  if (cls != 0)
    return false;
  const uint64_t n = count();
  out.resize(n);
  for (uint64_t i = 0u; i < n; ++i) {
    uint64_t v = 0u;
    std::memcpy(&v, raw.data() + i * size, size);
    if (is_signed && size < 8u && (v >> (8u * size - 1u)))
      v |= ~0ull << (8u * size);
    out[i] = (int)(int64_t)v;
  }
  return true;
}

bool read(const std::string &file, const std::string &path, Array &out, std::string &err)
{
  Reader r;
  uint64_t oh;
  return r.open(file, err) && r.lookup(path, oh, err) && r.dataset(oh, out, nullptr, err);
}

bool exists(const std::string &file, const std::string &path, std::string &err)
{
  Reader r;
  uint64_t oh;
  if (!r.open(file, err))
    return false;
  return r.lookup(path, oh, err);
}

// ---------------------------------------------------------------------------
// write side (classic format: superblock v0, object headers v1, symbol-table
// groups with 8-byte offsets and lengths)
// ---------------------------------------------------------------------------
namespace {

constexpr unsigned kLeafK = 4u, kNodeK = 16u; // symbol table node / B-tree K
constexpr uint64_t kSbEof = 40u, kSbRoot = 56u;

struct Bytes {
  std::vector<uint8_t> b;
  Bytes &u(uint64_t v, unsigned n)
  {
    for (unsigned i = 0u; i < n; ++i)
      b.push_back((uint8_t)(v >> (8u * i)));
    return *this;
  }
  Bytes &raw(const void *p, size_t n)
  {
    const uint8_t *c = static_cast<const uint8_t *>(p);
    b.insert(b.end(), c, c + n);
    return *this;
  }
  Bytes &pad(size_t a)
  {
    while (b.size() % a)
      b.push_back(0u);
    return *this;
  }
  Bytes &zeros(size_t n)
  {
    b.insert(b.end(), n, 0u);
    return *this;
  }
};

class Out {
public:
  ~Out()
  {
    if (f_)
      std::fclose(f_);
  }
  bool open(const std::string &path, bool create, std::string &err)
  {
    f_ = std::fopen(path.c_str(), create ? "w+xb" : "r+b");
    if (!f_) {
      err = (create ? "cannot create " : "cannot open for writing ") + path;
      return false;
    }
    if (std::fseek(f_, 0, SEEK_END))
      return false;
    eof_ = (uint64_t)std::ftell(f_);
    return true;
  }
  bool put(uint64_t off, const void *p, size_t n)
  {
    return !std::fseek(f_, (long)off, SEEK_SET) && std::fwrite(p, 1, n, f_) == n;
  }
  bool put64(uint64_t off, uint64_t v)
  {
    Bytes b;
    b.u(v, 8);
    return put(off, b.b.data(), 8);
  }
  // append at the end, 8-byte aligned; returns the address or kUndef
  uint64_t append(const void *p, size_t n)
  {
    const uint64_t a = (eof_ + 7u) & ~7ull;
    if (a > eof_) {
      const uint8_t z[8] = {0};
      if (!put(eof_, z, a - eof_))
        return kUndef;
    }
    if (n && !put(a, p, n))
      return kUndef;
    eof_ = a + n;
    return a;
  }
  uint64_t append(const Bytes &b) { return append(b.b.data(), b.b.size()); }
  uint64_t eof() const { return eof_; }
  bool close_ok()
  {
    const bool ok = std::fflush(f_) == 0;
    const bool ok2 = std::fclose(f_) == 0;
    f_ = nullptr;
    return ok && ok2;
  }

private:
  FILE *f_ = nullptr;
  uint64_t eof_ = 0u;
};

struct HMsg {
  unsigned type, flags;
  Bytes data;
};

// object header, version 1
Bytes ohdr_v1(std::vector<HMsg> &ms)
{
  uint64_t body = 0u;
  for (HMsg &m : ms) {
    m.data.pad(8);
    body += 8u + m.data.b.size();
  }
  Bytes h;
  h.u(1, 1).u(0, 1).u(ms.size(), 2).u(1, 4).u(body, 4).u(0, 4);
  for (const HMsg &m : ms)
    h.u(m.type, 2).u(m.data.b.size(), 2).u(m.flags, 1).zeros(3).raw(m.data.b.data(), m.data.b.size());
  return h;
}

HMsg symtab_msg(uint64_t btree, uint64_t heap)
{
  HMsg m{0x11u, 0u, {}};
  m.data.u(btree, 8).u(heap, 8);
  return m;
}

// a group's symbol table: local heap, symbol table nodes, one B-tree node;
// returns (B-tree, heap) addresses
bool write_symtab(Out &o, std::vector<Entry> es, uint64_t &btree, uint64_t &heap, std::string &err)
{
  std::sort(es.begin(), es.end(), [](const Entry &a, const Entry &b) { return a.name < b.name; });
  for (size_t i = 1u; i < es.size(); ++i)
    if (es[i].name == es[i - 1u].name) {
      err = "duplicate name " + es[i].name;
      return false;
    }
  const size_t per = 2u * kLeafK;
  const size_t nodes = (es.size() + per - 1u) / per;
  if (nodes > 2u * kNodeK) {
    err = "too many objects in one group for this writer";
    return false;
  }
  Bytes hd; // heap data: "" at 0, then the names
  hd.zeros(8);
  std::vector<uint64_t> noff(es.size());
  for (size_t i = 0u; i < es.size(); ++i) {
    noff[i] = hd.b.size();
    hd.raw(es[i].name.data(), es[i].name.size()).u(0, 1).pad(8);
  }
  const uint64_t hda = o.append(hd);
  Bytes hh;
  hh.raw("HEAP", 4).u(0, 1).zeros(3).u(hd.b.size(), 8).u(kUndef, 8).u(hda, 8);
  heap = o.append(hh);
  std::vector<uint64_t> snod(nodes);
  for (size_t k = 0u; k < nodes; ++k) {
    Bytes s;
    const size_t lo = k * per, hi = std::min(es.size(), lo + per);
    s.raw("SNOD", 4).u(1, 1).u(0, 1).u(hi - lo, 2);
    for (size_t i = lo; i < hi; ++i)
      s.u(noff[i], 8).u(es[i].ohdr, 8).u(0, 4).u(0, 4).zeros(16);
    s.zeros((per - (hi - lo)) * 40u);
    snod[k] = o.append(s);
  }
  Bytes t;
  t.raw("TREE", 4).u(0, 1).u(0, 1).u(nodes, 2).u(kUndef, 8).u(kUndef, 8);
  t.u(0, 8); // key 0: the empty name
  for (size_t k = 0u; k < nodes; ++k) {
    const size_t last = std::min(es.size(), (k + 1u) * per) - 1u;
    t.u(snod[k], 8).u(noff[last], 8);
  }
  t.zeros((2u * kNodeK - nodes) * 16u);
  btree = o.append(t);
  if (hda == kUndef || heap == kUndef || btree == kUndef) {
    err = "write failed";
    return false;
  }
  return true;
}

bool fresh_file(const std::string &file, std::string &err)
{
  Out o;
  if (!o.open(file, true, err))
    return false;
  Bytes sb;
  sb.raw(kSig, 8).u(0, 1).u(0, 1).u(0, 1).u(0, 1).u(0, 1).u(8, 1).u(8, 1).u(0, 1);
  sb.u(kLeafK, 2).u(kNodeK, 2).u(0, 4);
  sb.u(0, 8).u(kUndef, 8).u(0, 8).u(kUndef, 8); // base, free space, end of file, driver
  sb.zeros(40);                                  // root symbol table entry, filled below
  if (o.append(sb) != 0u) {
    err = "write failed";
    return false;
  }
  uint64_t bt, hp;
  if (!write_symtab(o, {}, bt, hp, err))
    return false;
  std::vector<HMsg> ms;
  ms.push_back(symtab_msg(bt, hp));
  const uint64_t root = o.append(ohdr_v1(ms));
  Bytes ste;
  ste.u(0, 8).u(root, 8).u(1, 4).u(0, 4).u(bt, 8).u(hp, 8);
  if (root == kUndef || !o.put(kSbRoot, ste.b.data(), ste.b.size()) || !o.put64(kSbEof, o.eof()) || !o.close_ok()) {
    err = "write failed";
    return false;
  }
  return true;
}

Bytes dataset_ohdr(const NewDataset &d, uint64_t data_addr, uint64_t nbytes)
{
  std::vector<HMsg> ms;
  HMsg sp{0x01u, 0u, {}};
  sp.data.u(1, 1).u(d.dims.size(), 1).u(1, 1).zeros(5);
  for (uint64_t x : d.dims)
    sp.data.u(x, 8);
  for (uint64_t x : d.dims)
    sp.data.u(x, 8);
  ms.push_back(sp);
  HMsg ty{0x03u, 1u, {}};
  if (d.is_float) // IEEE binary64, little endian, implied leading mantissa bit, sign at bit 63
    ty.data.u(0x11, 1).u(0x20, 1).u(63, 1).u(0, 1).u(8, 4).u(0, 2).u(64, 2).u(52, 1).u(11, 1).u(0, 1).u(52, 1).u(1023,
                                                                                                                 4);
  else // 32-bit two's complement, little endian
    ty.data.u(0x10, 1).u(0x08, 1).u(0, 1).u(0, 1).u(4, 4).u(0, 2).u(32, 2);
  ms.push_back(ty);
  HMsg fv{0x05u, 1u, {}};
  fv.data.u(2, 1).u(2, 1).u(2, 1).u(0, 1); // version 2, late allocation, fill if set, no fill value
  ms.push_back(fv);
  HMsg ly{0x08u, 0u, {}};
  ly.data.u(3, 1).u(1, 1).u(data_addr, 8).u(nbytes, 8); // version 3, contiguous
  ms.push_back(ly);
  return ohdr_v1(ms);
}

uint64_t elems(const std::vector<uint64_t> &dims)
{
  uint64_t c = 1u;
  for (uint64_t x : dims)
    c *= x;
  return c;
}

} // namespace

bool write_group(const std::string &file, const std::string &group, const std::vector<NewDataset> &ds, int mode,
                 std::string &err)
{
  if (group.empty() || group.find('/') != std::string::npos) {
    err = "group must be one name below the root";
    return false;
  }
  for (const NewDataset &d : ds)
    if (d.name.empty() || d.name.find('/') != std::string::npos || !d.data) {
      err = "bad dataset " + d.name;
      return false;
    }
  struct stat st;
  const bool there = stat(file.c_str(), &st) == 0;
  if (mode == 0) {
    if (there) {
      err = file + " exists";
      return false;
    }
    if (!fresh_file(file, err))
      return false;
  }
  else if (!there) {
    err = file + " does not exist";
    return false;
  }

  // everything we need from the existing file, before writing to it
  std::vector<Entry> root_es, grp_es;
  SymTab root_st, grp_st;
  uint64_t grp_oh = kUndef;
  struct Old {
    uint64_t addr;
    Array a;
  };
  std::vector<Old> old(ds.size(), Old{kUndef, {}});
  {
    Reader r;
    if (!r.open(file, err))
      return false;
    if (r.version() != 0u || r.so() != 8u || r.sl() != 8u || r.sb() != 0u) {
      err = "this writer adds only to classic-format files (superblock v0, 8-byte offsets)";
      return false;
    }
    std::vector<Msg> ms;
    if (!r.messages(r.root(), ms, err) || !r.symtab(ms, root_st)) {
      err = "root group has no symbol table";
      return false;
    }
    if (!r.entries(r.root(), root_es, err))
      return false;
    for (const Entry &e : root_es)
      if (e.name == group)
        grp_oh = e.ohdr;
    if (grp_oh != kUndef) {
      if (mode == 1) {
        err = "group " + group + " exists";
        return false;
      }
      if (!r.messages(grp_oh, ms, err) || !r.symtab(ms, grp_st)) {
        err = group + " is not a classic group";
        return false;
      }
      if (!r.entries(grp_oh, grp_es, err))
        return false;
      for (size_t i = 0u; i < ds.size(); ++i)
        for (const Entry &e : grp_es)
          if (e.name == ds[i].name) {
            if (!r.dataset(e.ohdr, old[i].a, &old[i].addr, err))
              return false;
            const Array &a = old[i].a;
            const bool same = a.dims == ds[i].dims && a.cls == (ds[i].is_float ? 1 : 0) &&
                              a.size == (ds[i].is_float ? 8u : 4u) && old[i].addr != kUndef;
            if (!same) {
              err = "dataset " + ds[i].name + " exists with another type or shape";
              return false;
            }
          }
    }
  }

  Out o;
  if (!o.open(file, false, err))
    return false;
  bool new_group = false;
  if (grp_oh == kUndef) { // an empty group, then linked into the root below
    uint64_t bt, hp;
    if (!write_symtab(o, {}, bt, hp, err))
      return false;
    std::vector<HMsg> ms;
    ms.push_back(symtab_msg(bt, hp));
    Bytes h = ohdr_v1(ms);
    grp_oh = o.append(h);
    grp_st.msg_off = grp_oh + 16u + 8u; // first message's data
    new_group = true;
  }
  bool added = false;
  for (size_t i = 0u; i < ds.size(); ++i) {
    const NewDataset &d = ds[i];
    const uint64_t nbytes = elems(d.dims) * (d.is_float ? 8u : 4u);
    if (old[i].addr != kUndef) { // overwrite in place
      if (!o.put(old[i].addr, d.data, nbytes)) {
        err = "write failed";
        return false;
      }
      continue;
    }
    const uint64_t da = o.append(d.data, nbytes);
    const uint64_t oh = o.append(dataset_ohdr(d, da, nbytes));
    if (da == kUndef || oh == kUndef) {
      err = "write failed";
      return false;
    }
    grp_es.push_back({d.name, oh});
    added = true;
  }
  if (added || new_group) {
    uint64_t bt, hp;
    if (!write_symtab(o, grp_es, bt, hp, err))
      return false;
    Bytes m;
    m.u(bt, 8).u(hp, 8);
    if (!o.put(grp_st.msg_off, m.b.data(), 16)) {
      err = "write failed";
      return false;
    }
  }
  if (new_group) {
    root_es.push_back({group, grp_oh});
    uint64_t bt, hp;
    if (!write_symtab(o, root_es, bt, hp, err))
      return false;
    Bytes m;
    m.u(bt, 8).u(hp, 8);
    Bytes cache;
    cache.u(1, 4).u(0, 4).u(bt, 8).u(hp, 8); // the superblock's cached copy
    if (!o.put(root_st.msg_off, m.b.data(), 16) || !o.put(kSbRoot + 16u, cache.b.data(), cache.b.size())) {
      err = "write failed";
      return false;
    }
  }
  if (!o.put64(kSbEof, o.eof()) || !o.close_ok()) {
    err = "write failed";
    return false;
  }
  return true;
}

} // namespace h5m
