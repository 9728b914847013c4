// YAML-subset reader and the fluid sections of config::loadConfig (src/IO/YamlConfig.cpp).
#include "YamlConfig.hpp"

#include <cctype>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace config {

const Node *Node::get(const std::string &key) const {
  if (kind != Map) return nullptr;
  auto it = children.find(key);
  return it == children.end() ? nullptr : it->second.get();
}

namespace {

std::string trim(const std::string &s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

// Removes a trailing comment (a '#' outside quotes that starts the line or follows a space).
std::string strip_comment(const std::string &s) {
  char quote = 0;
  for (size_t i = 0; i < s.size(); ++i) {
    const char c = s[i];
    if (quote) {
      if (c == quote) quote = 0;
    } else if (c == '"' || c == '\'') {
      quote = c;
    } else if (c == '#' && (i == 0 || std::isspace((unsigned char)s[i - 1]))) {
      return s.substr(0, i);
    }
  }
  return s;
}

std::string unquote(const std::string &s) {
  if (s.size() >= 2 && ((s.front() == '"' && s.back() == '"') || (s.front() == '\'' && s.back() == '\'')))
    return s.substr(1, s.size() - 2);
  return s;
}

struct Line {
  int indent;
  std::string text;
  int number;
};

std::runtime_error error(int line, const std::string &what) {
  return std::runtime_error("YAML line " + std::to_string(line) + ": " + what);
}

// Parses the block mapping whose keys sit at indentation `indent`, starting at lines[pos].
std::shared_ptr<Node> parse_map(const std::vector<Line> &lines, size_t &pos, int indent) {
  auto node = std::make_shared<Node>();
  node->kind = Node::Map;
  while (pos < lines.size()) {
    const Line &ln = lines[pos];
    if (ln.indent < indent) break;
    if (ln.indent > indent) throw error(ln.number, "unexpected indentation");
    const size_t colon = ln.text.find(':');
    if (colon == std::string::npos) throw error(ln.number, "expected 'key: value'");
    const std::string key = unquote(trim(ln.text.substr(0, colon)));
    const std::string rest = trim(ln.text.substr(colon + 1));
    if (key.empty()) throw error(ln.number, "empty key");
    if (node->children.count(key)) throw error(ln.number, "duplicate key '" + key + "'");
    ++pos;
    if (rest.empty()) {
      if (pos < lines.size() && lines[pos].indent > indent) {
        node->children[key] = parse_map(lines, pos, lines[pos].indent);
      } else {
        auto empty = std::make_shared<Node>();
        empty->kind = Node::Scalar;
        node->children[key] = empty;
      }
    } else if (rest.front() == '[') {
      if (rest.back() != ']') throw error(ln.number, "unterminated flow sequence");
      auto seq = std::make_shared<Node>();
      seq->kind = Node::Sequence;
      const std::string body = rest.substr(1, rest.size() - 2);
      std::stringstream ss(body);
      std::string item;
      while (std::getline(ss, item, ',')) {
        item = trim(item);
        if (!item.empty()) seq->items.push_back(unquote(item));
      }
      node->children[key] = seq;
    } else {
      auto sc = std::make_shared<Node>();
      sc->kind = Node::Scalar;
      sc->scalar = unquote(rest);
      node->children[key] = sc;
    }
  }
  return node;
}

double as_double(const Node *n, const std::string &key) {
  if (n->kind != Node::Scalar) throw std::runtime_error("'" + key + "' must be a number");
  size_t used = 0;
  double v = 0.0;
  try {
    v = std::stod(n->scalar, &used);
  } catch (...) {
    used = 0;
  }
  if (used == 0 || used != n->scalar.size()) throw std::runtime_error("'" + key + "' must be a number");
  return v;
}
int as_int(const Node *n, const std::string &key) {
  const double v = as_double(n, key);
  if (v != (double)(int)v) throw std::runtime_error("'" + key + "' must be an integer");
  return (int)v;
}
bool as_bool(const Node *n, const std::string &key) {
  if (n->kind == Node::Scalar) {
    const std::string &s = n->scalar;
    if (s == "true" || s == "True" || s == "TRUE" || s == "yes" || s == "on") return true;
    if (s == "false" || s == "False" || s == "FALSE" || s == "no" || s == "off") return false;
  }
  throw std::runtime_error("'" + key + "' must be true or false");
}
Vec3 as_vec3(const Node *n, const std::string &key) {
  if (n->kind != Node::Sequence || n->items.size() != 3)
    throw std::runtime_error("Invalid Vector3d format - expected [x, y, z] for '" + key + "'");
  Vec3 v;
  for (int c = 0; c < 3; ++c) {
    Node t;
    t.kind = Node::Scalar;
    t.scalar = n->items[c];
    v[c] = as_double(&t, key);
  }
  return v;
}

template <class F>
void opt(const Node *sec, const char *key, F &&apply) {
  if (!sec) return;
  if (const Node *n = sec->get(key)) apply(n, std::string(key));
}

void one_of(const std::string &v, std::initializer_list<const char *> allowed, const std::string &key) {
  for (const char *a : allowed)
    if (v == a) return;
  throw std::runtime_error("unknown value '" + v + "' for '" + key + "'");
}

}  // namespace

std::shared_ptr<Node> parseYaml(const std::string &text) {
  std::vector<Line> lines;
  std::stringstream ss(text);
  std::string raw;
  int number = 0;
  while (std::getline(ss, raw)) {
    ++number;
    if (!raw.empty() && raw.back() == '\r') raw.pop_back();
    if (raw.find('\t') != std::string::npos && trim(strip_comment(raw)).size())
      for (char c : raw) {
        if (c == '\t') throw error(number, "tabs are not allowed for indentation");
        if (c != ' ') break;
      }
    const std::string body = strip_comment(raw);
    if (trim(body).empty()) continue;
    if (trim(body) == "---") continue;
    int indent = 0;
    while (indent < (int)body.size() && body[indent] == ' ') ++indent;
    lines.push_back({indent, trim(body), number});
  }
  size_t pos = 0;
  if (lines.empty()) return std::make_shared<Node>();
  auto root = parse_map(lines, pos, lines[0].indent);
  if (pos != lines.size()) throw error(lines[pos].number, "unexpected indentation");
  return root;
}

SimulationConfig parseConfig(const std::string &text) {
  auto root = parseYaml(text);
  SimulationConfig c;
  const Node *mesh = root->get("mesh");
  if (!mesh || mesh->kind != Node::Map) throw std::runtime_error("Mesh configuration is required");
  // mesh (src/IO/YamlConfig.cpp:30-66)
  {
    const Node *t = mesh->get("type");
    if (!t) throw std::runtime_error("Mesh type not specified");
    c.mesh.type = t->scalar;
    one_of(c.mesh.type, {"cylinder", "msh", "y_bifurcation"}, "mesh.type");
    opt(mesh, "length", [&](const Node *n, const std::string &k) { c.mesh.cylinder_length = as_double(n, k); });
    opt(mesh, "radius", [&](const Node *n, const std::string &k) { c.mesh.cylinder_radius = as_double(n, k); });
    opt(mesh, "divisions", [&](const Node *n, const std::string &k) { c.mesh.cylinder_divisions = as_int(n, k); });
    opt(mesh, "max_element_size", [&](const Node *n, const std::string &k) { c.mesh.max_element_size = as_double(n, k); });
    opt(mesh, "rings", [&](const Node *n, const std::string &k) { c.mesh.rings = as_int(n, k); });
    opt(mesh, "layers", [&](const Node *n, const std::string &k) { c.mesh.layers = as_int(n, k); });
    opt(mesh, "msh_file", [&](const Node *n, const std::string &) { c.mesh.msh_file = n->scalar; });
    opt(mesh, "cell", [&](const Node *n, const std::string &k) { c.mesh.cell = as_double(n, k); });
    opt(mesh, "flow_direction", [&](const Node *n, const std::string &k) { c.mesh.flow_direction = as_vec3(n, k); });
    opt(mesh, "inlet_outlet_coverage", [&](const Node *n, const std::string &k) { c.mesh.inlet_outlet_coverage = as_double(n, k); });
    if (c.mesh.type == "msh" && c.mesh.msh_file.empty()) throw std::runtime_error("msh_file required for msh mesh type");
  }
  // navier_stokes (src/IO/YamlConfig.cpp:68-96)
  const Node *ns = root->get("navier_stokes");
  if (ns && ns->kind == Node::Map) {
    opt(ns, "enabled", [&](const Node *n, const std::string &k) { c.navier_stokes.enabled = as_bool(n, k); });
    if (c.navier_stokes.enabled) {
      auto &N = c.navier_stokes;
      opt(ns, "density", [&](const Node *n, const std::string &k) { N.density = as_double(n, k); });
      opt(ns, "viscosity", [&](const Node *n, const std::string &k) { N.viscosity = as_double(n, k); });
      opt(ns, "is_newtonian", [&](const Node *n, const std::string &k) { N.is_newtonian = as_bool(n, k); });
      opt(ns, "is_laminar", [&](const Node *n, const std::string &k) { N.is_laminar = as_bool(n, k); });
      opt(ns, "inlet_velocity", [&](const Node *n, const std::string &k) { N.inlet_velocity = as_vec3(n, k); });
      opt(ns, "outlet_pressure", [&](const Node *n, const std::string &k) { N.outlet_pressure = as_double(n, k); });
      opt(ns, "use_dirichlet_pressure", [&](const Node *n, const std::string &k) { N.use_dirichlet_pressure = as_bool(n, k); });
      opt(ns, "dt", [&](const Node *n, const std::string &k) { N.dt = as_double(n, k); });
      opt(ns, "relax_p", [&](const Node *n, const std::string &k) { N.relax_p = as_double(n, k); });
      opt(ns, "relax_u", [&](const Node *n, const std::string &k) { N.relax_u = as_double(n, k); });
      opt(ns, "tolerance", [&](const Node *n, const std::string &k) { N.tolerance = as_double(n, k); });
      opt(ns, "n_corrections", [&](const Node *n, const std::string &k) { N.n_corrections = as_int(n, k); });
      opt(ns, "max_iterations", [&](const Node *n, const std::string &k) {
        if (n->kind == Node::Sequence && n->items.size() == 2) {
          for (int q = 0; q < 2; ++q) {
            Node t;
            t.kind = Node::Scalar;
            t.scalar = n->items[q];
            N.max_iterations[q] = as_int(&t, k);
          }
        } else {
          N.max_iterations[0] = N.max_iterations[1] = as_int(n, k);
        }
      });
      opt(ns, "precision", [&](const Node *n, const std::string &k) { N.precision = n->scalar; one_of(N.precision, {"fp64", "mixed", "mixed_full"}, k); });
      opt(ns, "pressure_solver", [&](const Node *n, const std::string &k) { N.pressure_solver = n->scalar; one_of(N.pressure_solver, {"bicgstab", "cg", "cg1", "cg2l"}, k); });
      opt(ns, "momentum_solver", [&](const Node *n, const std::string &k) { N.momentum_solver = n->scalar; one_of(N.momentum_solver, {"bicgstab", "cg"}, k); });
      opt(ns, "coarse_aggregates", [&](const Node *n, const std::string &k) {
        N.coarse_aggregates = as_int(n, k);
        if (N.coarse_aggregates < 1 || N.coarse_aggregates > 1024)
          throw std::runtime_error("navier_stokes.coarse_aggregates must be in [1, 1024]");
      });
      opt(ns, "convergence_norm", [&](const Node *n, const std::string &k) { N.convergence_norm = n->scalar; one_of(N.convergence_norm, {"reference", "jacobi"}, k); });
      opt(ns, "inlet_profile", [&](const Node *n, const std::string &k) { N.inlet_profile = n->scalar; one_of(N.inlet_profile, {"uniform", "parabolic"}, k); });
    }
  }
  // enabled flags of the sections this build does not run
  auto enabled = [&](const char *sec) {
    const Node *s = root->get(sec);
    const Node *e = s ? s->get("enabled") : nullptr;
    return e ? as_bool(e, std::string(sec) + ".enabled") : false;
  };
  c.solid_mechanics_enabled = enabled("solid_mechanics");
  c.dpm_enabled = enabled("dpm");
  c.fsi_enabled = enabled("fsi_coupling");
  // output (src/IO/YamlConfig.cpp:180-197)
  const Node *out = root->get("output");
  opt(out, "prefix", [&](const Node *n, const std::string &) { c.output.output_prefix = n->scalar; });
  opt(out, "total_steps", [&](const Node *n, const std::string &k) { c.output.total_steps = as_int(n, k); });
  opt(out, "output_frequency", [&](const Node *n, const std::string &k) { c.output.output_frequency = as_int(n, k); });
  opt(out, "vtk_scale", [&](const Node *n, const std::string &k) { c.output.vtk_scale = as_double(n, k); });
  opt(out, "output_fluid", [&](const Node *n, const std::string &k) { c.output.output_fluid = as_bool(n, k); });
  if (c.output.output_frequency < 1) throw std::runtime_error("output_frequency must be >= 1");
  // adjoint (new)
  const Node *adj = root->get("adjoint");
  opt(adj, "enabled", [&](const Node *n, const std::string &k) { c.adjoint.enabled = as_bool(n, k); });
  opt(adj, "objective", [&](const Node *n, const std::string &k) { c.adjoint.objective = n->scalar; one_of(c.adjoint.objective, {"wall_shear", "pressure_drop"}, k); });
  opt(adj, "axis", [&](const Node *n, const std::string &k) { c.adjoint.axis = as_int(n, k); });
  opt(adj, "lo", [&](const Node *n, const std::string &k) { c.adjoint.lo = as_double(n, k); });
  opt(adj, "hi", [&](const Node *n, const std::string &k) { c.adjoint.hi = as_double(n, k); });
  opt(adj, "checkpoint_every", [&](const Node *n, const std::string &k) { c.adjoint.checkpoint_every = as_int(n, k); });
  opt(adj, "output", [&](const Node *n, const std::string &) { c.adjoint.output = n->scalar; });
  return c;
}

SimulationConfig loadConfig(const std::string &yaml_file) {
  std::ifstream in(yaml_file);
  if (!in.is_open()) throw std::runtime_error("cannot open " + yaml_file);
  std::stringstream ss;
  ss << in.rdbuf();
  return parseConfig(ss.str());
}

std::string describe(const SimulationConfig &c) {
  std::ostringstream o;
  o.precision(17);
  const auto &M = c.mesh;
  const auto &N = c.navier_stokes;
  o << "mesh.type = " << M.type << "\nmesh.length = " << M.cylinder_length << "\nmesh.radius = " << M.cylinder_radius
    << "\nmesh.max_element_size = " << M.max_element_size << "\nmesh.rings = " << M.rings
    << "\nmesh.layers = " << M.layers << "\nmesh.msh_file = " << M.msh_file << "\nmesh.cell = " << M.cell
    << "\nmesh.flow_direction = " << M.flow_direction.x() << " " << M.flow_direction.y() << " " << M.flow_direction.z()
    << "\nmesh.inlet_outlet_coverage = " << M.inlet_outlet_coverage << "\nnavier_stokes.enabled = " << N.enabled
    << "\nnavier_stokes.density = " << N.density << "\nnavier_stokes.viscosity = " << N.viscosity
    << "\nnavier_stokes.inlet_velocity = " << N.inlet_velocity.x() << " " << N.inlet_velocity.y() << " "
    << N.inlet_velocity.z() << "\nnavier_stokes.outlet_pressure = " << N.outlet_pressure
    << "\nnavier_stokes.use_dirichlet_pressure = " << N.use_dirichlet_pressure << "\nnavier_stokes.dt = " << N.dt
    << "\nnavier_stokes.relax_p = " << N.relax_p << "\nnavier_stokes.relax_u = " << N.relax_u
    << "\nnavier_stokes.tolerance = " << N.tolerance << "\nnavier_stokes.max_iterations = " << N.max_iterations[0]
    << " " << N.max_iterations[1] << "\nnavier_stokes.n_corrections = " << N.n_corrections
    << "\nnavier_stokes.precision = " << N.precision << "\nnavier_stokes.pressure_solver = " << N.pressure_solver
    << "\nnavier_stokes.coarse_aggregates = " << N.coarse_aggregates
    << "\nnavier_stokes.momentum_solver = " << N.momentum_solver
    << "\nnavier_stokes.convergence_norm = " << N.convergence_norm << "\nnavier_stokes.inlet_profile = "
    << N.inlet_profile << "\noutput.prefix = " << c.output.output_prefix << "\noutput.total_steps = "
    << c.output.total_steps << "\noutput.output_frequency = " << c.output.output_frequency
    << "\noutput.vtk_scale = " << c.output.vtk_scale << "\noutput.output_fluid = " << c.output.output_fluid
    << "\nadjoint.enabled = " << c.adjoint.enabled << "\nadjoint.objective = " << c.adjoint.objective
    << "\nadjoint.axis = " << c.adjoint.axis << "\nadjoint.lo = " << c.adjoint.lo << "\nadjoint.hi = " << c.adjoint.hi
    << "\nadjoint.checkpoint_every = " << c.adjoint.checkpoint_every << "\nadjoint.output = " << c.adjoint.output
    << "\nsolid_mechanics.enabled = " << c.solid_mechanics_enabled << "\ndpm.enabled = " << c.dpm_enabled
    << "\nfsi_coupling.enabled = " << c.fsi_enabled << "\n";
  return o.str();
}

}  // namespace config
