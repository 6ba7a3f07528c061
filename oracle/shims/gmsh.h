// Test infrastructure only: a minimal stand-in for the Gmsh C++ API so that the
// reference solver's own translation units compile and run here (Gmsh is not
// installed).  It implements exactly the ten calls the reference makes
// (src/mesh.cpp:9-20,48,58,64,70,281-282) on top of a reader for ASCII
// MSH 2.2 files, with the ordering Gmsh exposes for a file loaded that way:
//   * getNodes(): every node, in ascending node tag order;
//   * getPhysicalGroups(): (dim, tag) pairs in ascending (dim, tag) order;
//   * getEntitiesForPhysicalGroup(): elementary tags in ascending order;
//   * getElements(dim, entity): element types in ascending type order, the
//     elements of one type in file order.
// Only the oracle build includes this header; the product has its own reader.
#ifndef O2F_ORACLE_GMSH_SHIM_H
#define O2F_ORACLE_GMSH_SHIM_H

#include <algorithm>
#include <array>
#include <cstddef>
#include <fstream>
#include <map>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace gmsh {
namespace detail {

struct Element {
  int type;
  int phys;
  int entity;
  std::vector<std::size_t> nodes;
};

struct Model {
  std::map<std::size_t, std::array<double, 3>> nodes;  // tag -> xyz
  std::map<std::pair<int, int>, std::string> names;    // (dim, tag) -> name
  std::vector<Element> elements;                       // file order
};

inline Model& state() {
  static Model m;
  return m;
}

inline int element_dim(int type) {
  switch (type) {
    case 15: return 0;
    case 1: return 1;
    case 2: case 3: return 2;
    default: return 3;
  }
}

inline int element_nodes(int type) {
  switch (type) {
    case 15: return 1;
    case 1: return 2;
    case 2: return 3;
    case 3: return 4;
    case 4: return 4;
    default: throw std::runtime_error("gmsh shim: unsupported element type " + std::to_string(type));
  }
}

}  // namespace detail

inline void initialize(int = 0, char** = nullptr, bool = true, bool = false) {}
inline void finalize() {}
inline void clear() { detail::state() = detail::Model(); }

namespace option {
inline void setNumber(const std::string&, const double) {}
}  // namespace option

// Binary variant of the same model, written by oracle/ref.py for large
// meshes: "O2FMSHB1", int64 n_nodes, n_nodes x (x,y,z) f64 (tags 1..n),
// int64 n_names, per name (int32 dim, int32 tag, int32 len, bytes), int64
// n_elements, int32 type/phys/entity per element, then the int64 node tags.
inline bool open_binary(const std::string& fileName) {
  using namespace detail;
  std::ifstream in(fileName, std::ios::binary);
  char magic[8] = {0};
  if (!in.read(magic, 8) || std::string(magic, 8) != "O2FMSHB1") return false;
  Model& m = state();
  int64_t n = 0;
  in.read(reinterpret_cast<char*>(&n), 8);
  std::vector<double> xyz(3 * n);
  in.read(reinterpret_cast<char*>(xyz.data()), 24 * n);
  for (int64_t i = 0; i < n; ++i) m.nodes[i + 1] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
  int64_t nn = 0;
  in.read(reinterpret_cast<char*>(&nn), 8);
  for (int64_t i = 0; i < nn; ++i) {
    int32_t d[3];
    in.read(reinterpret_cast<char*>(d), 12);
    std::string name(d[2], '\0');
    in.read(&name[0], d[2]);
    m.names[{d[0], d[1]}] = name;
  }
  int64_t ne = 0;
  in.read(reinterpret_cast<char*>(&ne), 8);
  std::vector<int32_t> hdr(3 * ne);
  in.read(reinterpret_cast<char*>(hdr.data()), 12 * ne);
  int64_t total = 0;
  for (int64_t i = 0; i < ne; ++i) total += element_nodes(hdr[3 * i]);
  std::vector<int64_t> tags(total);
  in.read(reinterpret_cast<char*>(tags.data()), 8 * total);
  if (!in) throw std::runtime_error("gmsh shim: truncated binary mesh " + fileName);
  m.elements.resize(ne);
  int64_t o = 0;
  for (int64_t i = 0; i < ne; ++i) {
    Element& e = m.elements[i];
    e.type = hdr[3 * i];
    e.phys = hdr[3 * i + 1];
    e.entity = hdr[3 * i + 2];
    e.nodes.assign(tags.begin() + o, tags.begin() + o + element_nodes(e.type));
    o += element_nodes(e.type);
  }
  return true;
}

inline void open(const std::string& fileName) {
  using namespace detail;
  Model& m = state();
  m = Model();
  if (open_binary(fileName)) return;
  std::ifstream in(fileName);
  if (!in) throw std::runtime_error("gmsh shim: cannot open " + fileName);
  std::string line;
  while (std::getline(in, line)) {
    if (line.rfind("$PhysicalNames", 0) == 0) {
      int n = 0;
      in >> n;
      for (int i = 0; i < n; ++i) {
        int dim, tag;
        std::string name;
        in >> dim >> tag;
        std::getline(in, name);
        auto a = name.find('"'), b = name.rfind('"');
        if (a != std::string::npos && b != std::string::npos && b > a) name = name.substr(a + 1, b - a - 1);
        m.names[{dim, tag}] = name;
      }
    } else if (line.rfind("$Nodes", 0) == 0) {
      std::size_t n = 0;
      in >> n;
      for (std::size_t i = 0; i < n; ++i) {
        std::size_t tag;
        double x, y, z;
        in >> tag >> x >> y >> z;
        m.nodes[tag] = {x, y, z};
      }
    } else if (line.rfind("$Elements", 0) == 0) {
      std::size_t n = 0;
      in >> n;
      m.elements.reserve(n);
      for (std::size_t i = 0; i < n; ++i) {
        std::size_t id;
        int type, ntags;
        in >> id >> type >> ntags;
        std::vector<int> tags(ntags);
        for (int k = 0; k < ntags; ++k) in >> tags[k];
        Element e;
        e.type = type;
        e.phys = ntags > 0 ? tags[0] : 0;
        e.entity = ntags > 1 ? tags[1] : 0;
        e.nodes.resize(element_nodes(type));
        for (auto& v : e.nodes) in >> v;
        m.elements.push_back(std::move(e));
      }
    }
  }
}

namespace model {

inline void getPhysicalGroups(std::vector<std::pair<int, int>>& dimTags, const int dim = -1) {
  using namespace detail;
  std::set<std::pair<int, int>> groups;
  for (const auto& e : state().elements) {
    int d = element_dim(e.type);
    if (e.phys != 0 && (dim < 0 || d == dim)) groups.insert({d, e.phys});
  }
  dimTags.assign(groups.begin(), groups.end());
}

inline void getPhysicalName(const int dim, const int tag, std::string& name) {
  auto it = detail::state().names.find({dim, tag});
  name = it == detail::state().names.end() ? std::string() : it->second;
}

inline void getEntitiesForPhysicalGroup(const int dim, const int tag, std::vector<int>& tags) {
  using namespace detail;
  std::set<int> ents;
  for (const auto& e : state().elements)
    if (element_dim(e.type) == dim && e.phys == tag) ents.insert(e.entity);
  tags.assign(ents.begin(), ents.end());
}

namespace mesh {

inline void getNodes(std::vector<std::size_t>& nodeTags, std::vector<double>& coord,
                     std::vector<double>& parametricCoord, const int = -1, const int = -1,
                     const bool = false, const bool = true) {
  nodeTags.clear();
  coord.clear();
  parametricCoord.clear();
  for (const auto& [tag, xyz] : detail::state().nodes) {
    nodeTags.push_back(tag);
    coord.insert(coord.end(), xyz.begin(), xyz.end());
  }
}

inline void getElements(std::vector<int>& elementTypes, std::vector<std::vector<std::size_t>>& elementTags,
                        std::vector<std::vector<std::size_t>>& nodeTags, const int dim = -1,
                        const int tag = -1) {
  using namespace detail;
  std::map<int, std::pair<std::vector<std::size_t>, std::vector<std::size_t>>> by_type;
  std::size_t counter = 0;
  for (const auto& e : state().elements) {
    ++counter;
    if (dim >= 0 && element_dim(e.type) != dim) continue;
    if (tag >= 0 && e.entity != tag) continue;
    auto& slot = by_type[e.type];
    slot.first.push_back(counter);
    slot.second.insert(slot.second.end(), e.nodes.begin(), e.nodes.end());
  }
  elementTypes.clear();
  elementTags.clear();
  nodeTags.clear();
  for (auto& [type, lists] : by_type) {
    elementTypes.push_back(type);
    elementTags.push_back(std::move(lists.first));
    nodeTags.push_back(std::move(lists.second));
  }
}

}  // namespace mesh
}  // namespace model
}  // namespace gmsh

#endif  // O2F_ORACLE_GMSH_SHIM_H
