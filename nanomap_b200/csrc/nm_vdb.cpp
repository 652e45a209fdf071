// nm_vdb.cpp -- active voxels of a grid in an OpenVDB .vdb file, for sim grids loaded the way
// SimManager::loadGridFromFile (SimManager.h:196-213) loads them: the float grid named "grid".
//
// Only what the sim cast needs is read: the grid's transform (voxel size, translation) and its
// tree topology (which voxels and tiles are active).  The value buffers that follow the
// topology are never touched, and the values stored inside the topology (internal-node tiles)
// are skipped by the sizes stored in front of them, so no zip or blosc decoding is needed.
//
// Layout read (OpenVDB file format versions 222-224: io/Archive, tree/RootNode,
// tree/InternalNode, tree/LeafNode, math/Maps; all little endian):
//   header:  int64 magic 0x56444220, uint32 version, uint32 library major, minor,
//            uint8 has-grid-offsets (must be 1), 36-byte UUID text
//   file metadata: uint32 count, then per entry name, type name (uint32 length + bytes) and
//            uint32 size + value bytes
//   int32 grid count; per grid: unique name, type name, instance parent name (strings), int64
//            grid, block and end offsets (absolute); the grid section starts at the grid offset:
//            uint32 compression flags, grid metadata (as above), transform (map type name,
//            then the map's doubles), topology
//   topology: int32 buffer count (1); root: background value, uint32 tile count, uint32 child
//            count, tiles (int32 xyz, value, uint8 active), children (int32 xyz, internal
//            node); internal node (32^3, then 16^3 children): child mask, value mask, the
//            node's tile values (compressed, below), then its children in child-mask order;
//            leaf (8^3): value mask
//   compressed values: uint8 per-node code (0-6), then 0-2 inactive values (full size), a
//            selection mask for codes 3-5, then the values: all of them, or only the active
//            ones (value mask count) when the grid's flags hold COMPRESS_ACTIVE_MASK (0x2)
//            and the code is not 6; stored raw, or behind an int64 byte count when the flags
//            hold COMPRESS_ZIP (0x1) or COMPRESS_BLOSC (0x4) (a count <= 0: -count raw bytes)
//   masks: 2^(3 log2dim) bits in 64-bit words; bit n of a node is local (x, y, z) with
//            n = (x << 2 log2dim) | (y << log2dim) | z
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "nanomap_b200.h"
#include "nm_objects.h"

namespace {

constexpr int64_t kVdbMagic = 0x56444220;
constexpr uint32_t kCompressZip = 0x1, kCompressActiveMask = 0x2, kCompressBlosc = 0x4;
constexpr int64_t kMaxVoxels = int64_t(1) << 28;  // host list of 12 B per voxel: 3 GiB

struct Reader {
  FILE* f = nullptr;
  std::string err;
  int code = NM_ERR_IO;  // status of the first error
  ~Reader() {
    if (f) std::fclose(f);
  }
  bool ok() const { return err.empty(); }
  bool fail(int c, std::string msg) {
    if (ok()) {
      code = c;
      err = std::move(msg);
    }
    return false;
  }
  bool bytes(void* dst, size_t n) {
    if (!ok()) return false;
    if (n && std::fread(dst, 1, n, f) != n) err = "file ends early";
    return ok();
  }
  bool skip(int64_t n) {
    if (!ok()) return false;
    if (n < 0 || fseeko(f, (off_t)n, SEEK_CUR) != 0) err = "bad skip";
    return ok();
  }
  bool seek(int64_t pos) {
    if (!ok()) return false;
    if (pos < 0 || fseeko(f, (off_t)pos, SEEK_SET) != 0) err = "bad offset";
    return ok();
  }
  template <class T>
  T get() {
    T v{};
    bytes(&v, sizeof(T));
    return v;
  }
  std::string str() {
    const uint32_t n = get<uint32_t>();
    if (!ok()) return {};
    if (n > (1u << 20)) {
      err = "string too long";
      return {};
    }
    std::string s(n, '\0');
    bytes(&s[0], n);
    return s;
  }
  // metadata map: every value is behind its byte size
  bool skip_meta() {
    const uint32_t count = get<uint32_t>();
    for (uint32_t i = 0; i < count && ok(); ++i) {
      str();
      str();
      const uint32_t size = get<uint32_t>();
      skip(size);
    }
    return ok();
  }
};

struct Mask {
  std::vector<uint64_t> w;
  explicit Mask(int log2dim) : w(((size_t)1 << (3 * log2dim)) / 64, 0) {}
  bool load(Reader& r) { return r.bytes(w.data(), w.size() * 8); }
  bool on(uint32_t n) const { return (w[n >> 6] >> (n & 63)) & 1u; }
  uint32_t count() const {
    uint32_t c = 0;
    for (uint64_t x : w) c += (uint32_t)__builtin_popcountll(x);
    return c;
  }
};

struct Grid {
  uint32_t compression = 0;
  size_t value_size = 4;  // bytes per value in the topology's tile arrays
  size_t stored_size = 4;  // bytes per stored value (2 when saved as half)
  int64_t n_voxels = 0;
  int32_t* out = nullptr;  // null: count only
  int64_t max_out = 0;
};

// Skips one node's compressed values (count values, `active` of them active).
bool skip_values(Reader& r, const Grid& g, uint32_t count, uint32_t active, int log2dim) {
  const int8_t code = r.get<int8_t>();
  if (!r.ok()) return false;
  if (code < 0 || code > 6) return r.fail(NM_ERR_IO, "bad value-compression code");
  if (code == 2 || code == 4 || code == 5) r.skip((int64_t)g.value_size);  // inactive value 0
  if (code == 5) r.skip((int64_t)g.value_size);                            // inactive value 1
  if (code >= 3 && code <= 5) r.skip((int64_t)Mask(log2dim).w.size() * 8);  // selection mask
  const uint32_t n = ((g.compression & kCompressActiveMask) && code != 6) ? active : count;
  const int64_t raw = (int64_t)n * (int64_t)g.stored_size;
  if (g.compression & (kCompressZip | kCompressBlosc)) {
    const int64_t stored = r.get<int64_t>();
    if (!r.ok()) return false;
    if (stored <= 0 && -stored != raw)
      return r.fail(NM_ERR_IO, "uncompressed chunk of unexpected size");
    return r.skip(stored <= 0 ? -stored : stored);
  }
  return r.skip(raw);
}

// Adds the active voxels of the cube [o, o + edge)^3.
bool emit_cube(Reader& r, Grid& g, const int32_t o[3], int edge) {
  const int64_t n = (int64_t)edge * edge * edge;
  if (g.n_voxels + n > kMaxVoxels)
    return r.fail(NM_ERR_CAPACITY, "more active voxels than this reader takes (2^28)");
  if (g.out)
    for (int x = 0; x < edge; ++x)
      for (int y = 0; y < edge; ++y)
        for (int z = 0; z < edge; ++z) {
          const int64_t i = g.n_voxels + ((int64_t)x * edge + y) * edge + z;
          if (i >= g.max_out) continue;
          g.out[3 * i] = o[0] + x;
          g.out[3 * i + 1] = o[1] + y;
          g.out[3 * i + 2] = o[2] + z;
        }
  g.n_voxels += n;
  return true;
}

bool read_leaf(Reader& r, Grid& g, const int32_t o[3]) {
  Mask vm(3);
  if (!vm.load(r)) return false;
  for (uint32_t n = 0; n < 512; ++n) {
    if (!vm.on(n)) continue;
    if (g.n_voxels + 1 > kMaxVoxels)
      return r.fail(NM_ERR_CAPACITY, "more active voxels than this reader takes (2^28)");
    if (g.out && g.n_voxels < g.max_out) {
      int32_t* v = g.out + 3 * g.n_voxels;
      v[0] = o[0] + (int32_t)(n >> 6);
      v[1] = o[1] + (int32_t)((n >> 3) & 7);
      v[2] = o[2] + (int32_t)(n & 7);
    }
    ++g.n_voxels;
  }
  return true;
}

// Internal node of 2^log2dim per axis whose children span 2^child_total voxels per axis
// (log2dim 5 over 4 over leaves: 4096 = 32 x 16 x 8 voxels per axis at the top).
bool read_internal(Reader& r, Grid& g, const int32_t o[3], int log2dim, int child_total) {
  Mask cm(log2dim), vm(log2dim);
  if (!cm.load(r) || !vm.load(r)) return false;
  const uint32_t count = 1u << (3 * log2dim);
  if (!skip_values(r, g, count, vm.count(), log2dim)) return false;
  const uint32_t dmask = (1u << log2dim) - 1u;
  auto origin = [&](uint32_t n, int32_t c[3]) {
    c[0] = o[0] + (int32_t)((n >> (2 * log2dim)) << child_total);
    c[1] = o[1] + (int32_t)(((n >> log2dim) & dmask) << child_total);
    c[2] = o[2] + (int32_t)((n & dmask) << child_total);
  };
  // active tiles (value-mask bits without a child)
  for (uint32_t n = 0; n < count; ++n) {
    if (!vm.on(n) || cm.on(n)) continue;
    int32_t c[3];
    origin(n, c);
    if (!emit_cube(r, g, c, 1 << child_total)) return false;
  }
  for (uint32_t n = 0; n < count && r.ok(); ++n) {
    if (!cm.on(n)) continue;
    int32_t c[3];
    origin(n, c);
    const bool ok = child_total == 3 ? read_leaf(r, g, c)
                                     : read_internal(r, g, c, 4, 3);
    if (!ok) return false;
  }
  return r.ok();
}

bool read_topology(Reader& r, Grid& g) {
  const int32_t buffers = r.get<int32_t>();
  if (r.ok() && buffers != 1) r.fail(NM_ERR_UNSUPPORTED, "multi-buffer tree");
  r.skip((int64_t)g.value_size);  // background
  const uint32_t tiles = r.get<uint32_t>(), children = r.get<uint32_t>();
  if (!r.ok()) return false;
  if (tiles > (1u << 24) || children > (1u << 24)) return r.fail(NM_ERR_IO, "implausible root table");
  for (uint32_t i = 0; i < tiles && r.ok(); ++i) {
    int32_t c[3];
    r.bytes(c, 12);
    r.skip((int64_t)g.value_size);
    const uint8_t active = r.get<uint8_t>();
    if (active && !emit_cube(r, g, c, 4096)) return false;
  }
  for (uint32_t i = 0; i < children && r.ok(); ++i) {
    int32_t c[3];
    r.bytes(c, 12);
    if (!read_internal(r, g, c, 5, 7)) return false;
  }
  return r.ok();
}

// Voxel size and translation of the index-to-world map.
bool read_transform(Reader& r, double vs[3], double tr[3]) {
  const std::string type = r.str();
  double v[18];
  tr[0] = tr[1] = tr[2] = 0.0;
  if (type == "UniformScaleMap" || type == "ScaleMap") {
    // scale, voxel size, inverse scale, inverse scale squared, inverse twice scale
    if (!r.bytes(v, 15 * 8)) return false;
    for (int a = 0; a < 3; ++a) vs[a] = v[3 + a];
  } else if (type == "UniformScaleTranslateMap" || type == "ScaleTranslateMap") {
    // translation, then as above
    if (!r.bytes(v, 18 * 8)) return false;
    for (int a = 0; a < 3; ++a) {
      tr[a] = v[a];
      vs[a] = v[6 + a];
    }
  } else if (type == "TranslationMap") {
    if (!r.bytes(v, 3 * 8)) return false;
    for (int a = 0; a < 3; ++a) {
      tr[a] = v[a];
      vs[a] = 1.0;
    }
  } else if (type == "AffineMap") {
    // 4x4 row-major, row vectors: scale on the diagonal, translation in the last row
    double m[16];
    if (!r.bytes(m, sizeof(m))) return false;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        if (i != j && m[4 * i + j] != 0.0)
          return r.fail(NM_ERR_UNSUPPORTED, "rotated or sheared AffineMap");
    for (int a = 0; a < 3; ++a) {
      vs[a] = m[5 * a];
      tr[a] = m[12 + a];
    }
  } else {
    return r.fail(NM_ERR_UNSUPPORTED, "transform '" + type + "' is not a scale and translation");
  }
  return r.ok();
}

}  // namespace

int nm_vdb_active_voxels(const char* path, const char* grid, double voxel_size[3],
                         double translation[3], int32_t* ijk, int64_t max_voxels, int64_t* n) {
  if (!path || !n || (ijk && max_voxels < 0)) return nm::fail(NM_ERR_ARG, "invalid argument");
  *n = 0;
  Reader r;
  r.f = std::fopen(path, "rb");
  if (!r.f) return nm::fail(NM_ERR_IO, "cannot open '%s'", path);
  const int64_t magic = r.get<int64_t>();
  const uint32_t version = r.get<uint32_t>();
  if (!r.ok() || magic != kVdbMagic) return nm::fail(NM_ERR_IO, "%s: not an OpenVDB file", path);
  if (version < 222 || version > 224)
    return nm::fail(NM_ERR_UNSUPPORTED, "%s: OpenVDB file format %u (this reader takes 222-224)",
                    path, version);
  r.get<uint32_t>();  // library major
  r.get<uint32_t>();  // library minor
  const uint8_t offsets = r.get<uint8_t>();
  r.skip(36);  // UUID
  if (r.ok() && offsets != 1)
    return nm::fail(NM_ERR_UNSUPPORTED, "%s: grids stored without offsets (a stream, not a file)",
                    path);
  r.skip_meta();
  const int32_t grids = r.get<int32_t>();
  if (!r.ok() || grids < 0 || grids > (1 << 20))
    return nm::fail(NM_ERR_IO, "%s: %s", path, r.ok() ? "bad grid count" : r.err.c_str());
  const std::string want = grid ? grid : "grid";
  int64_t pos = -1;
  std::string type, first_type, names;
  int64_t first_pos = -1;
  for (int32_t i = 0; i < grids && r.ok(); ++i) {
    std::string name = r.str();
    const std::string t = r.str();
    r.str();  // instance parent
    const int64_t gpos = r.get<int64_t>();
    r.get<int64_t>();  // block offset
    const int64_t end = r.get<int64_t>();
    // a unique name is the grid name, then 0x1E and a number for repeated names
    const size_t cut = name.find('\x1e');
    if (cut != std::string::npos) name.resize(cut);
    if (!names.empty()) names += ", ";
    names += name;
    if (i == 0) {
      first_pos = gpos;
      first_type = t;
    }
    if (pos < 0 && name == want) {
      pos = gpos;
      type = t;
    }
    r.seek(end);
  }
  if (!r.ok()) return nm::fail(NM_ERR_IO, "%s: %s", path, r.err.c_str());
  if (pos < 0) {
    if (grid || first_pos < 0)
      return nm::fail(NM_ERR_ARG, "%s: no grid named '%s' (grids: %s)", path, want.c_str(),
                      names.c_str());
    pos = first_pos;  // no "grid" and no name asked for: the file's first grid
    type = first_type;
  }
  Grid g;
  const std::string half = "_HalfFloat";
  bool as_half = false;
  if (type.size() > half.size() && type.compare(type.size() - half.size(), half.size(), half) == 0) {
    as_half = true;
    type.resize(type.size() - half.size());
  }
  if (type == "Tree_float_5_4_3") {
    g.value_size = 4;
    g.stored_size = as_half ? 2 : 4;
  } else if (type == "Tree_double_5_4_3") {
    g.value_size = 8;
    g.stored_size = as_half ? 2 : 8;
  } else {
    return nm::fail(NM_ERR_UNSUPPORTED, "%s: grid type %s (this reader takes float and double 5-4-3 trees)",
                    path, type.c_str());
  }
  r.seek(pos);
  g.compression = r.get<uint32_t>();
  r.skip_meta();
  double vs[3] = {0, 0, 0}, tr[3] = {0, 0, 0};
  if (!r.ok() || !read_transform(r, vs, tr)) return nm::fail(r.code, "%s: %s", path, r.err.c_str());
  g.out = ijk;
  g.max_out = ijk ? max_voxels : 0;
  if (!read_topology(r, g)) return nm::fail(r.code, "%s: %s", path, r.err.c_str());
  if (voxel_size) std::memcpy(voxel_size, vs, sizeof(vs));
  if (translation) std::memcpy(translation, tr, sizeof(tr));
  *n = g.n_voxels;
  if (ijk && g.n_voxels > max_voxels)
    return nm::fail(NM_ERR_CAPACITY, "%s: %lld active voxels, room for %lld", path,
                    (long long)g.n_voxels, (long long)max_voxels);
  return NM_OK;
}

// ---- writer: the same layout, for sim grids of active voxels --------------------------------
namespace {

struct Out {
  std::vector<unsigned char> b;
  template <class T>
  void put(const T& v) {
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
    b.insert(b.end(), p, p + sizeof(T));
  }
  void raw(const void* p, size_t n) {
    const unsigned char* q = static_cast<const unsigned char*>(p);
    b.insert(b.end(), q, q + n);
  }
  void str(const std::string& s) {
    put<uint32_t>((uint32_t)s.size());
    raw(s.data(), s.size());
  }
  void meta(const std::string& name, const std::string& type, const void* v, uint32_t n) {
    str(name);
    str(type);
    put<uint32_t>(n);
    raw(v, n);
  }
};

struct LeafMask {
  uint64_t w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

// A node's values: code 0 (every inactive value is the background), then the active values
// only (the grid is written with COMPRESS_ACTIVE_MASK), all 0.
void put_values(Out& o, uint32_t active) {
  o.put<int8_t>(0);
  for (uint32_t i = 0; i < active; ++i) o.put<float>(0.0f);
}

}  // namespace

int nm_vdb_write_active_voxels(const char* path, const char* grid, double voxel_size,
                               const int32_t* ijk, int64_t n) {
  if (!path || (n > 0 && !ijk) || n < 0) return nm::fail(NM_ERR_ARG, "invalid argument");
  if (!(voxel_size > 0.0) || !std::isfinite(voxel_size))
    return nm::fail(NM_ERR_ARG, "voxel size must be positive");
  // leaves by origin; the tree's order below comes from sorting origins by the nodes' offsets
  std::map<std::array<int32_t, 3>, LeafMask> leaves;
  for (int64_t i = 0; i < n; ++i) {
    const int32_t x = ijk[3 * i], y = ijk[3 * i + 1], z = ijk[3 * i + 2];
    LeafMask& m = leaves[{x & ~7, y & ~7, z & ~7}];
    const uint32_t bit = (uint32_t)(((x & 7) << 6) | ((y & 7) << 3) | (z & 7));
    m.w[bit >> 6] |= uint64_t(1) << (bit & 63);
  }
  // root children (32^3 nodes, 4096 voxels) -> their 16^3 children by offset -> leaves by offset
  std::map<std::array<int32_t, 3>, std::map<uint32_t, std::map<uint32_t, const LeafMask*>>> tree;
  for (const auto& kv : leaves) {
    const auto& o = kv.first;
    const std::array<int32_t, 3> r = {o[0] & ~4095, o[1] & ~4095, o[2] & ~4095};
    const uint32_t n5 = (uint32_t)((((o[0] - r[0]) >> 7) << 10) | (((o[1] - r[1]) >> 7) << 5) |
                                   ((o[2] - r[2]) >> 7));
    const int32_t i4[3] = {o[0] & ~127, o[1] & ~127, o[2] & ~127};
    const uint32_t n4 = (uint32_t)((((o[0] - i4[0]) >> 3) << 8) | (((o[1] - i4[1]) >> 3) << 4) |
                                   ((o[2] - i4[2]) >> 3));
    tree[r][n5][n4] = &kv.second;
  }
  const uint32_t compression = kCompressActiveMask;
  Out topo;
  topo.put<int32_t>(1);     // buffer count
  topo.put<float>(0.0f);    // background
  topo.put<uint32_t>(0);    // root tiles
  topo.put<uint32_t>((uint32_t)tree.size());
  std::vector<const LeafMask*> order;  // leaves in the order the buffers follow
  for (const auto& r : tree) {
    topo.raw(r.first.data(), 12);
    std::vector<uint64_t> cm5(512, 0);
    for (const auto& c : r.second) cm5[c.first >> 6] |= uint64_t(1) << (c.first & 63);
    topo.raw(cm5.data(), 4096);
    std::vector<uint64_t> vm5(512, 0);
    topo.raw(vm5.data(), 4096);
    put_values(topo, 0);
    for (const auto& c : r.second) {
      std::vector<uint64_t> cm4(64, 0), vm4(64, 0);
      for (const auto& l : c.second) cm4[l.first >> 6] |= uint64_t(1) << (l.first & 63);
      topo.raw(cm4.data(), 512);
      topo.raw(vm4.data(), 512);
      put_values(topo, 0);
      for (const auto& l : c.second) {
        topo.raw(l.second->w, 64);
        order.push_back(l.second);
      }
    }
  }
  Out buffers;
  for (const LeafMask* m : order) {
    buffers.raw(m->w, 64);
    uint32_t active = 0;
    for (uint64_t w : m->w) active += (uint32_t)__builtin_popcountll(w);
    put_values(buffers, active);
  }
  const std::string name = grid ? grid : "grid";
  Out head;
  head.put<int64_t>(kVdbMagic);
  head.put<uint32_t>(224);  // file format version
  head.put<uint32_t>(0);    // library version major, minor: not written by the OpenVDB library
  head.put<uint32_t>(0);
  head.put<uint8_t>(1);     // grids stored with offsets
  const char uuid[] = "6e6d2d62-3230-302d-7669-6d2d61637469";
  head.raw(uuid, 36);
  head.put<uint32_t>(0);  // no file metadata
  head.put<int32_t>(1);   // one grid
  head.str(name);
  head.str("Tree_float_5_4_3");
  head.str("");  // not an instance
  Out sec;
  sec.put<uint32_t>(compression);
  const char cls[] = "unknown";
  int32_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  if (n > 0)
    for (int a = 0; a < 3; ++a) {
      lo[a] = hi[a] = ijk[a];
      for (int64_t i = 1; i < n; ++i) {
        lo[a] = std::min(lo[a], ijk[3 * i + a]);
        hi[a] = std::max(hi[a], ijk[3 * i + a]);
      }
    }
  sec.put<uint32_t>(3);
  sec.meta("class", "string", cls, (uint32_t)std::strlen(cls));
  sec.meta("file_bbox_min", "vec3i", lo, 12);
  sec.meta("file_bbox_max", "vec3i", hi, 12);
  sec.str("UniformScaleMap");
  const double v = voxel_size, iv = 1.0 / voxel_size;
  const double map[15] = {v, v, v, v, v, v, iv, iv, iv, iv * iv, iv * iv, iv * iv,
                          iv / 2, iv / 2, iv / 2};
  sec.raw(map, sizeof(map));
  const int64_t grid_pos = (int64_t)head.b.size() + 24;
  const int64_t block_pos = grid_pos + (int64_t)sec.b.size() + (int64_t)topo.b.size();
  const int64_t end_pos = block_pos + (int64_t)buffers.b.size();
  head.put<int64_t>(grid_pos);
  head.put<int64_t>(block_pos);
  head.put<int64_t>(end_pos);
  FILE* f = std::fopen(path, "wb");
  if (!f) return nm::fail(NM_ERR_IO, "cannot write '%s'", path);
  bool ok = true;
  for (const Out* part : {&head, &sec, &topo, &buffers})
    ok = ok && (part->b.empty() || std::fwrite(part->b.data(), 1, part->b.size(), f) == part->b.size());
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return nm::fail(NM_ERR_IO, "short write to '%s'", path);
  return NM_OK;
}
