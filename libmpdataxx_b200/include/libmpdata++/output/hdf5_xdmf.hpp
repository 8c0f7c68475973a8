// output::hdf5_xdmf<solver_t> (libmpdata++/output/hdf5_xdmf.hpp, output/hdf5.hpp,
// output/detail/output_common.hpp, output/detail/xdmf_writer.hpp): the solver
// type with output.  concurr::cuda runs it like the plain solver and, on every
// output step (timestep % outfreq == 0, timestep >= outstart), reads the
// outvars back from the GPU -- the only device-to-host traffic -- and writes
//
//   <outdir>/const.h5               X, Y[, Z] cell-corner coordinates (float32,
//                                   grid + 1), T (the output times), group
//                                   "advection" (opts, dt, di, dj[, dk], var_dt, n_iters)
//   <outdir>/timestepNNNNNNNNNN.h5  one float32 dataset per output variable
//   <outdir>/timestepNNNNNNNNNN.xmf and <outdir>/temp.xmf   (XDMF)
//
// HDF5 is written by the small writer below, from the HDF5 file-format
// specification (superblock version 0, version-1 object headers, the root
// group as a symbol table, contiguous datasets): no HDF5 library is needed.
// Message encodings are the ones the HDF5 library writes for the reference;
// datasets are contiguous where the reference chunks and deflates them.  The
// XDMF text is the reference's byte for byte.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include <sys/stat.h>

#include <mpdx.h>

namespace libmpdataxx {
namespace output {
namespace detail {

class h5_writer {
 public:
  // root dataset: float32 data of the given shape (C order)
  void add_dataset(const std::string &name, const std::vector<float> &data, const std::vector<uint64_t> &shape) {
    ds_.push_back({name, data, shape});
  }
  // group of scalar attributes: value kinds 's' string, 'f' float32, 'i' int32, 'b' bool
  struct attr { std::string name; char kind; std::string s; double v; };
  void add_group(const std::string &name, const std::vector<attr> &attrs) { gr_.push_back({name, attrs}); }

  void write(const std::string &path) {
    b_.assign(96, 0);
    struct member { std::string name; uint64_t hdr; bool group; uint64_t btree, heap; };
    std::vector<member> ms;
    for (auto &d : ds_) ms.push_back({d.name, dataset(d), false, 0, 0});
    for (auto &g : gr_) {
      uint64_t hdr, bt, hp;
      group({}, g.attrs, hdr, bt, hp);
      ms.push_back({g.name, hdr, true, bt, hp});
    }
    std::sort(ms.begin(), ms.end(), [](const member &a, const member &b) { return a.name < b.name; });
    std::vector<link> links;
    for (auto &m : ms) links.push_back({m.name, m.hdr, m.group, m.btree, m.heap});
    uint64_t hdr, bt, hp;
    group(links, {}, hdr, bt, hp);
    std::string sb("\x89HDF\r\n\x1a\n", 8);
    sb += std::string("\0\0\0\0\0\x08\x08\0", 8);
    sb += u(4, 2) + u(16, 2) + u(0, 4) + u(0, 8) + u(kUndef, 8) + u(b_.size(), 8) + u(kUndef, 8);
    sb += u(0, 8) + u(hdr, 8) + u(1, 4) + u(0, 4) + u(bt, 8) + u(hp, 8);
    std::memcpy(b_.data(), sb.data(), sb.size());
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f) throw std::runtime_error("libmpdata++: cannot open " + path);
    f.write(reinterpret_cast<const char *>(b_.data()), std::streamsize(b_.size()));
  }

 private:
  static constexpr uint64_t kUndef = ~uint64_t(0);
  static constexpr int kLeafK = 4, kInternalK = 16;
  static constexpr size_t kBtree = 24 + (2 * kInternalK + 1) * 8 + 2 * kInternalK * 8, kSnod = 8 + 2 * kLeafK * 40;
  struct ds { std::string name; std::vector<float> data; std::vector<uint64_t> shape; };
  struct grp { std::string name; std::vector<attr> attrs; };
  struct link { std::string name; uint64_t hdr; bool group; uint64_t btree, heap; };
  std::vector<ds> ds_;
  std::vector<grp> gr_;
  std::vector<unsigned char> b_;

  static std::string u(uint64_t v, int n) {
    std::string s(size_t(n), '\0');
    for (int q = 0; q < n; ++q) s[size_t(q)] = char((v >> (8 * q)) & 0xff);
    return s;
  }
  static std::string pad8(std::string s) { s.resize((s.size() + 7) / 8 * 8, '\0'); return s; }
  uint64_t alloc(size_t n) {
    b_.resize((b_.size() + 7) / 8 * 8, 0);
    const uint64_t a = b_.size();
    b_.resize(b_.size() + n, 0);
    return a;
  }
  void put(uint64_t a, const std::string &s) { std::memcpy(b_.data() + a, s.data(), s.size()); }

  static std::string dataspace(const std::vector<uint64_t> &shape) {  // version 1, with maximum dimensions
    std::string s;
    s += char(1); s += char(shape.size()); s += char(1); s += char(0);
    s += u(0, 4);
    for (auto n : shape) s += u(n, 8);
    for (auto n : shape) s += u(n, 8);
    return s;
  }
  static std::string f32type() {  // IEEE float32 little-endian
    return std::string("\x11\x20\x1f\x00", 4) + u(4, 4) + u(0, 2) + u(32, 2) + std::string("\x17\x08\x00\x17", 4) + u(127, 4);
  }
  static std::string inttype(int bytes, bool is_signed) {
    std::string s;
    s += char(0x10); s += char(is_signed ? 0x08 : 0x00); s += char(0); s += char(0);
    return s + u(uint64_t(bytes), 4) + u(0, 2) + u(uint64_t(8 * bytes), 2);
  }
  static std::string message(int type, const std::string &data) {
    const std::string d = pad8(data);
    std::string s = u(uint64_t(type), 2) + u(d.size(), 2);
    s += std::string(4, '\0');
    return s + d;
  }
  static std::string object_header(const std::vector<std::string> &msgs) {
    std::string body;
    for (auto &m : msgs) body += m;
    std::string s;
    s += char(1); s += char(0);
    return s + u(msgs.size(), 2) + u(1, 4) + u(body.size(), 4) + u(0, 4) + body;
  }
  static std::string attribute(const attr &a) {
    const std::string nm = a.name + std::string(1, '\0');
    std::string type, data;
    if (a.kind == 's') { type = std::string("\x13\x00\x00\x00", 4) + u(a.s.size(), 4); data = a.s; }
    else if (a.kind == 'b') { type = inttype(1, false); data = u(a.v != 0 ? 1 : 0, 1); }
    else if (a.kind == 'i') { type = inttype(4, true); data = u(uint64_t(int64_t(a.v)) & 0xffffffffu, 4); }
    else { type = f32type(); const float f = float(a.v); uint32_t w; std::memcpy(&w, &f, 4); data = u(w, 4); }
    const std::string space = dataspace({1});
    std::string s;
    s += char(1); s += char(0);
    s += u(nm.size(), 2) + u(type.size(), 2) + u(space.size(), 2);
    return s + pad8(nm) + pad8(type) + pad8(space) + data;
  }
  uint64_t dataset(const ds &d) {
    const size_t bytes = d.data.size() * sizeof(float);
    const uint64_t at = alloc(bytes);
    std::memcpy(b_.data() + at, d.data.data(), bytes);
    const std::string fill("\x02\x01\x02\x01\x00\x00\x00\x00", 8);
    const std::string layout = std::string("\x03\x01", 2) + u(at, 8) + u(bytes, 8);
    const std::string h = object_header({message(0x01, dataspace(d.shape)), message(0x03, f32type()),
                                         message(0x05, fill), message(0x08, layout)});
    const uint64_t a = alloc(h.size());
    put(a, h);
    return a;
  }
  void group(const std::vector<link> &links, const std::vector<attr> &attrs, uint64_t &hdr, uint64_t &bt, uint64_t &hp) {
    if (links.size() > size_t(2 * kLeafK)) throw std::runtime_error("libmpdata++: too many output variables");
    std::string names(8, '\0');
    std::vector<uint64_t> offs;
    for (auto &l : links) { offs.push_back(names.size()); names += pad8(l.name + std::string(1, '\0')); }
    hp = alloc(32);
    const uint64_t data = alloc(names.size());
    put(data, names);
    put(hp, std::string("HEAP\0\0\0\0", 8) + u(names.size(), 8) + u(kUndef, 8) + u(data, 8));
    bt = alloc(kBtree);
    std::string node = std::string("TREE\0\0", 6) + u(links.empty() ? 0 : 1, 2) + u(kUndef, 8) + u(kUndef, 8);
    if (!links.empty()) {
      const uint64_t snod = alloc(kSnod);
      std::string e = std::string("SNOD\x01\x00", 6) + u(links.size(), 2);
      for (size_t q = 0; q < links.size(); ++q) {
        e += u(offs[q], 8) + u(links[q].hdr, 8);
        if (links[q].group) e += u(1, 4) + u(0, 4) + u(links[q].btree, 8) + u(links[q].heap, 8);
        else e += u(0, 4) + u(0, 4) + std::string(16, '\0');
      }
      put(snod, e);
      node += u(0, 8) + u(snod, 8) + u(offs.back(), 8);
    }
    put(bt, node);
    std::vector<std::string> msgs{message(0x11, u(bt, 8) + u(hp, 8))};
    for (auto &a : attrs) msgs.push_back(message(0x0C, attribute(a)));
    const std::string h = object_header(msgs);
    hdr = alloc(h.size());
    put(hdr, h);
  }
};

inline std::string dims(const std::vector<int> &d) {
  std::string s;
  for (int n : d) s += std::to_string(n) + " ";
  return s;
}

// XDMF of one record (xdmf_writer.hpp write(): boost::property_tree, one-tab indentation)
inline std::string xmf_record(const std::string &hdf, double time, const std::vector<int> &grid,
                              const std::vector<std::string> &vars, const std::string &cnst = "const.h5") {
  const int nd = int(grid.size());
  std::vector<int> corner;
  for (int n : grid) corner.push_back(n + 1);
  std::string s = "<?xml version=\"1.0\" encoding=\"utf-8\"?>\n<Xdmf>\n\t<Domain>\n";
  s += "\t\t<Grid Name=\"Grid\" GridType=\"Uniform\" xml:id=\"gid\">\n";
  s += "\t\t\t<Time Value=\"" + std::to_string(time) + "\"/>\n";
  s += "\t\t\t<Topology TopologyType=\"" + std::string(nd == 2 ? "2DSMesh" : "3DSMesh") + "\" Dimensions=\"" + dims(corner) + "\"/>\n";
  s += "\t\t\t<Geometry GeometryType=\"" + std::string(nd == 2 ? "X_Y" : "X_Y_Z") + "\">\n";
  const char *axes[3] = {"X", "Y", "Z"};
  for (int d = 0; d < nd; ++d)
    s += "\t\t\t\t<DataItem Dimensions=\"" + dims(corner) + "\" NumberType=\"Float\" Format=\"HDF\">" + cnst + ":/" + axes[d] + "</DataItem>\n";
  s += "\t\t\t</Geometry>\n";
  std::vector<std::string> sorted(vars);
  std::sort(sorted.begin(), sorted.end());
  for (auto &v : sorted) {
    s += "\t\t\t<Attribute Name=\"" + v + "\" AttributeType=\"Scalar\" Center=\"Cell\">\n";
    s += "\t\t\t\t<DataItem Dimensions=\"" + dims(grid) + "\" NumberType=\"Float\" Format=\"HDF\">" + hdf + ":/" + v + "</DataItem>\n";
    s += "\t\t\t</Attribute>\n";
  }
  return s + "\t\t</Grid>\n\t</Domain>\n</Xdmf>\n";
}

inline std::string xmf_temporal(const std::vector<std::string> &xmfs) {
  std::string s = "<?xml version=\"1.0\" encoding=\"utf-8\"?>\n<Xdmf xmlns:xi=\"http://www.w3.org/2001/XInclude\">\n";
  s += "\t<Domain>\n\t\t<Grid Name=\"TimeGrid\" GridType=\"Collection\" CollectionType=\"Temporal\">\n";
  for (auto &x : xmfs) s += "\t\t\t<xi:include href=\"" + x + "\" xpointer=\"gid\"/>\n";
  return s + "\t\t</Grid>\n\t</Domain>\n</Xdmf>\n";
}

inline void write_text(const std::string &path, const std::string &text) {
  std::ofstream f(path, std::ios::trunc);
  if (!f) throw std::runtime_error("libmpdata++: cannot open " + path);
  f << text;
}

// the writer behind output::hdf5_xdmf: const.h5 at start, one record per output step
class xdmf_recorder {
 public:
  xdmf_recorder(std::string outdir, std::vector<int> grid, double dt, std::vector<double> dijk,
                std::string opts_str, int n_iters)
      : dir_(std::move(outdir)), grid_(std::move(grid)), dt_(dt), dijk_(std::move(dijk)),
        opts_(std::move(opts_str)), n_iters_(n_iters) {}

  void start(const std::vector<double> &times) {
    ::mkdir(dir_.c_str(), 0755);
    const int nd = int(grid_.size());
    std::vector<uint64_t> shape;
    size_t n = 1;
    for (int g : grid_) { shape.push_back(uint64_t(g + 1)); n *= size_t(g + 1); }
    h5_writer w;
    const char *axes[3] = {"X", "Y", "Z"};
    for (int d = 0; d < nd; ++d) {
      std::vector<float> c(n);
      for (size_t q = 0; q < n; ++q) {
        size_t r = q;
        for (int e = nd - 1; e > d; --e) r /= size_t(grid_[size_t(e)] + 1);
        c[q] = float(dijk_[size_t(d)] * double(r % size_t(grid_[size_t(d)] + 1)));
      }
      w.add_dataset(axes[d], c, shape);
    }
    std::vector<float> t;
    for (double v : times) t.push_back(float(v));
    w.add_dataset("T", t, {uint64_t(t.size())});
    std::vector<h5_writer::attr> at{{"opts", 's', opts_, 0}, {"dt", 'f', "", dt_}};
    const char *dn[3] = {"di", "dj", "dk"};
    for (int d = 0; d < nd; ++d) at.push_back({dn[d], 'f', "", dijk_[size_t(d)]});
    at.push_back({"var_dt", 'b', "", 0});
    at.push_back({"n_iters", 'i', "", double(n_iters_)});
    w.add_group("advection", at);
    w.write(dir_ + "/const.h5");
  }

  // fields: name -> float32 values of the grid (C order)
  void record(long long timestep, const std::map<std::string, std::vector<float>> &fields) {
    char base[32];
    std::snprintf(base, sizeof base, "timestep%010lld", timestep);
    h5_writer w;
    std::vector<uint64_t> shape(grid_.begin(), grid_.end());
    std::vector<std::string> names;
    for (auto &f : fields) { w.add_dataset(f.first, f.second, shape); names.push_back(f.first); }
    w.write(dir_ + "/" + base + ".h5");
    write_text(dir_ + "/" + base + ".xmf", xmf_record(std::string(base) + ".h5", double(timestep) * dt_, grid_, names));
    xmfs_.push_back(std::string(base) + ".xmf");
    write_text(dir_ + "/temp.xmf", xmf_temporal(xmfs_));
  }

 private:
  std::string dir_;
  std::vector<int> grid_;
  double dt_;
  std::vector<double> dijk_;
  std::string opts_;
  int n_iters_;
  std::vector<std::string> xmfs_;
};

}  // namespace detail

// output::hdf5_xdmf<slv_t>: the solver type plus the output parameters of
// output_common.hpp:171-178 (outfreq, outstart, outvars, outdir)
template <class solver_t>
struct hdf5_xdmf : solver_t {
  static constexpr bool has_output = true;
  static_assert(solver_t::n_dims > 1, "only 2D and 3D output supported");  // hdf5_xdmf.hpp:38
  struct info_t { std::string name, unit; };
  struct rt_params_t : solver_t::rt_params_t {
    int outfreq = 1, outstart = 0;
    std::map<int, info_t> outvars;
    std::string outdir;
  };
  static void fill(mpdx_config &c, const rt_params_t &p) { solver_t::fill(c, p); }
};

}  // namespace output
}  // namespace libmpdataxx
