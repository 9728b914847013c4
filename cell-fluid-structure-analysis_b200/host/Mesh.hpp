// Tetrahedral mesh with P1 vertices, P2 edge nodes and fluid boundary tags.
//
// Host-side mirror of the reference Mesh class (include/Mesh/Mesh.hpp:15-220,
// src/Mesh/Mesh.cpp). Public names, argument meaning and the numbering rules the solver
// depends on are the same:
//   * faces are ordered by their sorted vertex triple (the reference keeps them in a
//     std::map keyed on that triple, src/Mesh/Mesh.cpp:496-530);
//   * P2 edge nodes are numbered in first-encounter order over tets and local edges
//     (0-1,0-2,0-3,1-2,1-3,2-3) (src/Mesh/Mesh.cpp:641-677); P2 global index = nv + edge id;
//   * boundary tagging walks faces in that order with last-write-wins
//     (src/Mesh/Mesh.cpp:325-417) and P2 tags follow include/Mesh/Mesh.hpp:198-215.
// The builds use sorting and bucketing instead of std::map so that multi-million-tet meshes
// are processed in seconds; the resulting orders are identical.
//
// TetGen-based constructors (fromObjFile/fromPolyhedron) are not provided: TetGen is not a
// dependency of this library. Meshes come from MSH 4.1 files, from arrays, from the structured
// prism generator, or from the procedural cylinder generator (Mesh::cylinder).
#pragma once

#include "FluidTypes.hpp"
#include "Vec3.hpp"

#include <array>
#include <cassert>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

struct Tet {
  double volume = 0.0;
  std::array<int, 4> vertids{};
  std::array<int, 4> faceids = {-1, -1, -1, -1};
  std::array<int, 4> neighbors = {-1, -1, -1, -1};
  Vec3 centroid = Vec3(0, 0, 0);
};

// Y-bifurcation: a parent tube of radius parent_radius along +x from x = 0 to parent_length
// splits into two daughter tubes (radius daughter_radius, length daughter_length) at angles
// +-angle_deg in the x-y plane, joined by a smooth union of blend radius `blend`. Meshed on a
// Kuhn-subdivided cubic lattice of edge `cell` (6 tets per cube, conforming), tets kept where
// the signed distance at their centroid is negative, wall vertices moved onto the surface and
// outlet vertices onto the cut planes when no tet around them degenerates. Tags: inlet on the
// x = 0 cap, outlet on both daughter caps, wall elsewhere (tilted outlets cannot be tagged by the
// axis-extreme rule of setupBoundaryConditions).
struct YBifurcation {
  double parent_radius = 2.0, parent_length = 15.0;
  double daughter_radius = 1.5, daughter_length = 12.0, angle_deg = 35.0;
  double blend = 0.5;
  double cell = 0.0813;  // lattice edge; about 4M tets at the defaults
};

struct Face {
  bool is_ecm = false;
  int tet_a = -1;
  int tet_b = -1;
  int face_id_a = -1;
  int face_id_b = -1;
  double area = 0.0;
  std::array<int, 3> vertids{};
  Vec3 normal = Vec3(0, 0, 0);
  Vec3 center;
};

class Mesh {
  double min_edge_length_ = 0.0;
  std::vector<Vec3> vertices_;    // P1 nodes
  std::vector<Vec3> edge_nodes_;  // P2 nodes (edge midpoints)
  std::vector<Face> faces_;
  std::vector<Tet> tets_;
  std::vector<std::vector<int>> vertex_neighbors_;
  std::vector<FluidBCType> p1_fluid_vert_bc_types_;
  std::vector<FluidBCType> p2_fluid_vert_bc_types_;
  std::vector<SolidBCType> solid_vert_bc_types_;
  std::vector<std::array<Vec3, 4>> tet_gradients_;
  // Edge (min vertex, max vertex) -> edge node id, sorted by key (replaces the std::map).
  std::vector<std::pair<std::pair<int, int>, int>> edge_to_node_id_;
  std::vector<std::array<int, 6>> tet_edge_nodes_;

  void finalizeFromArrays(bool check_degenerate);
  void buildVertexNeighbors();
  void buildConnectivity();
  void computeShapeFunctionGradients();
  void ensureConsistentFaceNormals();
  void buildP2EdgeNodes();
  void computeMinEdgeLength();
  bool hasDegenerateTet() const;

 public:
  Mesh() = default;

  void generateFromMshFile(const std::string &filename);
  void generateFromArrays(const std::vector<Vec3> &vertices,
                          const std::vector<std::array<int, 4>> &tets);
  void generateStructuredRectangularPrism(double length, double width, double height, int nx,
                                          int ny, int nz);
  // Procedural cylinder along +x: length L, radius R, centred on y = z = 0. The disk
  // cross-section has `rings` concentric rings (ring k has 6k points) and the axis is cut
  // into `layers` prism layers; each prism is split into 3 tets conformingly.
  void generateCylinder(double length, double radius, int rings, int layers);
  // Procedural Y-bifurcation with generator-assigned fluid tags (see YBifurcation).
  void generateYBifurcation(const struct YBifurcation &spec);
  void computeGeometry();

  static Mesh fromMshFile(const std::string &filename) {
    Mesh m;
    m.generateFromMshFile(filename);
    return m;
  }
  static Mesh fromArrays(const std::vector<Vec3> &vertices,
                         const std::vector<std::array<int, 4>> &tets) {
    Mesh m;
    m.generateFromArrays(vertices, tets);
    return m;
  }
  static Mesh structuredRectangularPrism(double length, double width, double height, int nx = 1,
                                         int ny = 1, int nz = 1) {
    Mesh m;
    m.generateStructuredRectangularPrism(length, width, height, nx, ny, nz);
    return m;
  }
  static Mesh cylinder(double length, double radius, int rings, int layers) {
    Mesh m;
    m.generateCylinder(length, radius, rings, layers);
    return m;
  }
  static Mesh yBifurcation(const YBifurcation &spec) {
    Mesh m;
    m.generateYBifurcation(spec);
    return m;
  }
  static void setupBoundaryConditions(const Vec3 &inlet_to_outlet_direction,
                                      double percent_inlet_to_outlet_converage, Mesh &mesh);

  // Writes the P1 mesh as Gmsh MSH 4.1 (one node block, one tet block), readable by
  // generateFromMshFile and by the reference's reader (src/Mesh/Mesh.cpp:16-144).
  void writeMshFile(const std::string &filename) const;

  bool isInitialized() { return !vertices_.empty() && !tets_.empty(); }
  void updateGeometry() {
    computeGeometry();
    computeShapeFunctionGradients();
  }

  // sizes
  size_t nVertices() const { return vertices_.size(); }
  size_t nTets() const { return tets_.size(); }
  size_t nFaces() const { return faces_.size(); }

  // getters
  const std::vector<Tet> &getTets() const { return tets_; }
  const Tet &tetAt(size_t tetidx) const {
    assert(tetidx < tets_.size());
    return tets_[tetidx];
  }
  Tet &tetAt(size_t tetidx) {
    assert(tetidx < tets_.size());
    return tets_[tetidx];
  }
  const std::array<int, 6> &getTetEdgeNodes(size_t ti) const {
    assert(ti < tet_edge_nodes_.size());
    return tet_edge_nodes_[ti];
  }
  const std::vector<std::array<int, 6>> &getAllTetEdgeNodes() const { return tet_edge_nodes_; }
  const std::vector<Face> &getFaces() const { return faces_; }
  const Face &faceAt(size_t faceidx) const {
    assert(faceidx < faces_.size());
    return faces_[faceidx];
  }
  Face &faceAt(size_t faceidx) {
    assert(faceidx < faces_.size());
    return faces_[faceidx];
  }
  const std::vector<Vec3> &getVertPositions() const { return vertices_; }
  const Vec3 &getVertexPositon(size_t vertid) const {
    assert(vertid < vertices_.size());
    return vertices_[vertid];
  }
  Vec3 &getVertexPositon(size_t vertid) {
    assert(vertid < vertices_.size());
    return vertices_[vertid];
  }
  const std::vector<Vec3> &getEdgeNodePositions() const { return edge_nodes_; }
  FluidBCType getFluidVertexBC(size_t vertex_id) const {
    assert(vertex_id < p1_fluid_vert_bc_types_.size());
    return p1_fluid_vert_bc_types_[vertex_id];
  }
  FluidBCType getP2FluidVertexBC(size_t p2_id) const {
    assert(p2_id < p2_fluid_vert_bc_types_.size());
    return p2_fluid_vert_bc_types_[p2_id];
  }
  SolidBCType getSolidVertexBC(size_t vid) const {
    assert(vid < solid_vert_bc_types_.size());
    return solid_vert_bc_types_[vid];
  }
  const std::vector<int> &getVertexNeighborInds(size_t vi) const {
    assert(vi < vertices_.size());
    return vertex_neighbors_[vi];
  }
  const Vec3 &getP2NodesAtEdge(size_t vi, size_t vj) const;
  int getEdgeNodeId(int vi, int vj) const;  // -1 if (vi,vj) is not an edge
  size_t getNumberOfEdgeNodes() const { return edge_nodes_.size(); }
  size_t getP1plusP2DegreesOfFreedom() const { return edge_nodes_.size() + vertices_.size(); }
  const std::array<Vec3, 4> &getTetGradient(size_t ti) const {
    assert(ti < tet_gradients_.size());
    return tet_gradients_[ti];
  }
  const std::array<Vec3, 4> &getTetGradients(size_t ti) const {
    assert(ti < tet_gradients_.size());
    return tet_gradients_[ti];
  }
  double getMinEdgeLength() const { return min_edge_length_; }

  // setters
  void setFluidVertexBC(size_t vertex_id, const FluidBCType bc_type) {
    if (p1_fluid_vert_bc_types_.empty()) {
      p1_fluid_vert_bc_types_.resize(vertices_.size(), FluidBCType::Undefined);
    }
    assert(vertex_id < p1_fluid_vert_bc_types_.size());
    p1_fluid_vert_bc_types_[vertex_id] = bc_type;
  }
  void setFluidP2vertexBC(size_t p2_id, const FluidBCType bc_type) {
    assert(p2_id < p2_fluid_vert_bc_types_.size());
    p2_fluid_vert_bc_types_[p2_id] = bc_type;
  }
  void setSolidVertexBC(size_t vid, const SolidBCType bc_type) {
    if (solid_vert_bc_types_.empty()) {
      solid_vert_bc_types_.resize(vertices_.size(), SolidBCType::Undefined);
    }
    assert(vid < solid_vert_bc_types_.size());
    solid_vert_bc_types_[vid] = bc_type;
  }
  // P2 node tag: the endpoints' common tag when both agree and are not Internal, else Internal
  // (include/Mesh/Mesh.hpp:198-215).
  void setP2BoundariesFromP1Boundaries();
  bool isFaceInternal(size_t fi) const {
    assert(fi < faces_.size());
    return faces_[fi].tet_b != -1;
  }
};
