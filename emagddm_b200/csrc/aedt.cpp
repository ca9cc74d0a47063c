// aedt.cpp -- material, object and boundary definitions of an Ansys Maxwell
// project file (.aedt, text), the data the reference's AedtProjectLoader
// takes from MaxwellParserImpl (src/tool/aedt_project_loader.cpp:60-130:
// parseMaterials, parseBoundaries; src/tool/maxwell_parser_impl.cpp) that the
// edge-element solve path needs: per material the relative permeability and
// the conductivity, per geometry part (object) its material, and the
// boundaries with their type and value.  The mesh itself is not in an .aedt
// file; a Gmsh mesh whose physical volumes carry the objects' names takes its
// nu / sigma from here (emagddm_b200.aedt).
//
// The file is a tree of `$begin 'Name'` ... `$end 'Name'` blocks holding
// `key=value` lines (values single-quoted when they are strings, numbers
// possibly followed by a unit), call-like lines (`Objects(12)`, `set(...)`)
// and arrays (`Points[4: h0, b0, h1, b1]`).  Materials are the children of
// Definitions/Materials: `permeability='1.05'` (relative) or a
// `$begin 'permeability'` block with property_type='nonlinear' and a BH
// curve (BHCoordinates/Points, pairs H [A/m], B [T]), whose initial
// permeability (the first point with H > 0: B / (mu0 H)) stands for it in a
// linear solve; `conductivity='58000000'` [S/m].  Objects are the GeometryPart
// blocks: Attributes/Name and Attributes/MaterialValue ('"copper"').
// Boundaries are the children of a Boundaries block: BoundType and Value.
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include "internal.h"

namespace emg {

namespace {

constexpr double kMu0 = 4e-7 * 3.14159265358979323846;

struct Node {
  std::string name;
  std::vector<std::pair<std::string, std::string>> values;  // key=value lines, in order
  std::vector<std::string> lines;                           // other lines
  std::vector<std::unique_ptr<Node>> children;
  Node* parent = nullptr;
  const std::string* get(const std::string& key) const {
    for (const auto& kv : values)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
  const Node* child(const std::string& n) const {
    for (const auto& c : children)
      if (c->name == n) return c.get();
    return nullptr;
  }
};

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace(static_cast<unsigned char>(s[a]))) ++a;
  while (b > a && std::isspace(static_cast<unsigned char>(s[b - 1]))) --b;
  return s.substr(a, b - a);
}

// 'abc' -> abc, '"abc"' -> abc
std::string unquote(std::string v) {
  v = trim(v);
  for (int pass = 0; pass < 2; ++pass) {
    if (v.size() >= 2 && ((v.front() == '\'' && v.back() == '\'') || (v.front() == '"' && v.back() == '"')))
      v = v.substr(1, v.size() - 2);
  }
  return v;
}

// Leading number of a value ('58000000', '1.05', '0mm'); NaN when none.
double number(const std::string& v) {
  const std::string s = unquote(v);
  const char* b = s.c_str();
  char* e = nullptr;
  const double x = std::strtod(b, &e);
  return e == b ? std::nan("") : x;
}

bool parse_tree(const std::string& path, Node& root, std::string& err) {
  std::ifstream f(path);
  if (!f) { err = "cannot open " + path; return false; }
  Node* cur = &root;
  std::string raw;
  int64_t lineno = 0;
  while (std::getline(f, raw)) {
    ++lineno;
    const std::string line = trim(raw);
    if (line.empty()) continue;
    if (line.rfind("$begin", 0) == 0) {
      auto n = std::make_unique<Node>();
      n->name = unquote(line.substr(6));
      n->parent = cur;
      cur->children.push_back(std::move(n));
      cur = cur->children.back().get();
    } else if (line.rfind("$end", 0) == 0) {
      if (!cur->parent || unquote(line.substr(4)) != cur->name) {
        err = "line " + std::to_string(lineno) + ": unbalanced block end '" + unquote(line.substr(4)) + "'";
        return false;
      }
      cur = cur->parent;
    } else {
      size_t eq = line.find('=');
      size_t k = 0;
      while (k < line.size() && (std::isalnum(static_cast<unsigned char>(line[k])) || line[k] == '_')) ++k;
      if (eq != std::string::npos && eq == k && k > 0) cur->values.emplace_back(line.substr(0, k), line.substr(eq + 1));
      else cur->lines.push_back(line);
    }
  }
  if (cur != &root) { err = "unterminated block '" + cur->name + "'"; return false; }
  return true;
}

void find_all(const Node& n, const std::string& name, std::vector<const Node*>& out) {
  for (const auto& c : n.children) {
    if (c->name == name) out.push_back(c.get());
    find_all(*c, name, out);
  }
}

// Points[n: a, b, c, ...] -> numbers
std::vector<double> array_values(const Node& n, const std::string& key) {
  std::vector<double> v;
  for (const std::string& l : n.lines) {
    if (l.rfind(key + "[", 0) != 0) continue;
    const size_t colon = l.find(':');
    size_t p = colon == std::string::npos ? key.size() + 1 : colon + 1;
    const char* s = l.c_str();
    while (p < l.size()) {
      char* e = nullptr;
      const double x = std::strtod(s + p, &e);
      if (e == s + p) { ++p; continue; }
      v.push_back(x);
      p = static_cast<size_t>(e - s);
    }
  }
  return v;
}

}  // namespace

int aedt_read(const std::string& path, AedtProject& out) {
  Node root;
  std::string err;
  if (!parse_tree(path, root, err)) { set_error("AEDT: " + err); return EMG_INVALID_INPUT; }
  std::vector<const Node*> defs;
  find_all(root, "Definitions", defs);
  const Node* mats = nullptr;
  for (const Node* d : defs)
    if ((mats = d->child("Materials"))) break;
  if (mats) {
    for (const auto& m : mats->children) {
      AedtProject::Material M;
      M.name = m->name;
      if (const std::string* v = m->get("permeability")) {
        M.mu_r = number(*v);
        if (std::isnan(M.mu_r)) M.flags |= 2;
      } else if (const Node* p = m->child("permeability")) {
        const std::string* t = p->get("property_type");
        if (t && unquote(*t) == "nonlinear") {
          M.flags |= 1;
          if (const Node* bh = p->child("BHCoordinates")) {
            const std::vector<double> pts = array_values(*bh, "Points");
            for (size_t i = 0; i + 1 < pts.size(); i += 2) { M.h.push_back(pts[i]); M.b.push_back(pts[i + 1]); }
          }
          M.mu_r = std::nan("");
          for (size_t i = 0; i < M.h.size(); ++i)
            if (M.h[i] > 0.0 && M.b[i] > 0.0) { M.mu_r = M.b[i] / (kMu0 * M.h[i]); break; }
          if (std::isnan(M.mu_r)) M.flags |= 2;
        } else if (const std::string* v2 = p->get("Magnitude")) {
          M.mu_r = number(*v2);
          if (std::isnan(M.mu_r)) M.flags |= 2;
        }
      }
      if (const std::string* v = m->get("conductivity")) {
        M.sigma = number(*v);
        if (std::isnan(M.sigma)) M.flags |= 4;
      }
      out.materials.push_back(std::move(M));
    }
  }
  std::vector<const Node*> parts;
  find_all(root, "GeometryPart", parts);
  for (const Node* g : parts) {
    const Node* a = g->child("Attributes");
    if (!a) continue;
    AedtProject::Object O;
    if (const std::string* v = a->get("Name")) O.name = unquote(*v);
    if (const std::string* v = a->get("MaterialValue")) O.material = unquote(*v);
    if (const std::string* v = a->get("SolveInside")) O.solve_inside = trim(*v) == "false" ? 0 : 1;
    out.objects.push_back(std::move(O));
  }
  std::vector<const Node*> bnds;
  find_all(root, "Boundaries", bnds);
  for (const Node* bs : bnds)
    for (const auto& bc : bs->children) {
      AedtProject::Boundary B;
      B.name = bc->name;
      if (const std::string* v = bc->get("BoundType")) B.type = unquote(*v);
      if (const std::string* v = bc->get("Value")) B.value = unquote(*v);
      out.boundaries.push_back(std::move(B));
    }
  return EMG_SUCCESS;
}

}  // namespace emg
