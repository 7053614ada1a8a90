// Host-side unstructured finite-volume mesh: connectivity, geometry, periodic pairing and
// least-squares gradient stencils.  This is the set-up the reference performs in Fortran before
// the time loop (src/mesh/mod_mesh.f90, src/mesh/mod_gmsh_reader.f90, src/bc/mod_bc_setup.f90);
// it is restated here so that a host without a Fortran toolchain can build the static operator
// data that the sm_100a time step consumes.  All indices are 0-based; "no cell" is -1.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace dpm {

// Boundary-condition ids (src/mod_parameters.f90:41-51).
enum BcId : int {
  BC_INLET = 1, BC_OUTLET = 2, BC_WALL_NOSLIP = 3, BC_WALL_MODEL = 4, BC_SLIP = 5,
  BC_PERIODIC = 6, BC_SYMMETRY = 7, BC_FIXEDTEMP = 8, BC_ZEROGRADIENT = 9,
  BC_WALL_VELOCITY = 10, BC_ABL_INLET = 11
};

// gmsh element type codes (src/mesh/mod_gmsh_reader.f90:14-23).
enum ElemType : int { EL_TRI3 = 2, EL_QUAD4 = 3, EL_TET4 = 4, EL_HEX8 = 5, EL_PRISM6 = 6, EL_PYR5 = 7 };

constexpr double SMALL = 1.0e-30;            // src/mod_parameters.f90:29
constexpr double REFINE_SKEW_TOL = 0.15;     // src/mesh/mod_mesh.f90:26
constexpr double SKEW_BLEND_LO = 0.15;       // src/mesh/mod_mesh.f90:30
constexpr double SKEW_BLEND_HI = 0.25;       // src/mesh/mod_mesh.f90:31
constexpr double LS_DET_TOL = 1.0e-12;       // src/mesh/mod_mesh.f90:19
constexpr double LS_REG_FRAC = 1.0e-6;       // src/mesh/mod_mesh.f90:20

// Raw mesh as a gmsh v4 file carries it: nodes, volume elements in file order, surface
// elements tagged with a physical-surface (patch) index.
struct RawMesh {
  int64_t n_nodes = 0;
  const double* xyz = nullptr;           // [n_nodes][3]
  int64_t n_cells = 0;
  const int* cell_type = nullptr;        // [n_cells] ElemType
  const int64_t* cell_off = nullptr;     // [n_cells+1]
  const int* cell_nodes = nullptr;       // node ids, gmsh local ordering
  int64_t n_bfaces = 0;
  const int64_t* bface_off = nullptr;    // [n_bfaces+1]
  const int* bface_nodes = nullptr;
  const int* bface_patch = nullptr;      // [n_bfaces] patch index 0..n_patches-1
  int n_patches = 0;
};

struct Mesh {
  int64_t n_cells = 0, n_faces = 0, n_int_faces = 0, n_bnd_faces = 0;
  int n_patches = 0;
  // cells
  std::vector<double> centroid;          // [nc][3]
  std::vector<double> volume;            // [nc]
  std::vector<int64_t> cell_face_off;    // [nc+1] CSR into cell_faces
  std::vector<int> cell_faces;           // face ids, in face order
  // faces (interior faces first, then boundary faces grouped by patch)
  std::vector<int> owner, neighbour;     // neighbour = -1 on boundary faces
  std::vector<int> patch;                // -1 on interior faces
  std::vector<double> area, centre, normal, sf;   // centre/normal/sf: [nf][3]
  std::vector<double> d_cf, gc, eps, skew;        // eps: [nf][3]
  std::vector<uint8_t> is_refine;
  // patches
  std::vector<int> patch_bc;             // [n_patches] BcId
  std::vector<int64_t> patch_start;      // boundary-face index of the first face of the patch
  std::vector<int64_t> patch_nfaces;
  // periodic pairing, indexed by boundary face (0..n_bnd-1); -1 = none
  std::vector<int> periodic_pair;
  std::vector<double> periodic_pair_dcf;
  std::vector<double> periodic_gc;       // owner weight of the periodic interpolation
  // vertex topology (for the vertex-neighbour LS stencil)
  int64_t n_vertices = 0;
  std::vector<double> vertices;          // [nv][3]
  std::vector<int64_t> cell_vert_off;    // [nc+1]
  std::vector<int> cell_vertices;
  // least-squares gradient stencil
  std::vector<int64_t> ls_off;           // [nc+1]
  std::vector<int> ls_cell;              // neighbour cell or -1 (boundary face-centre entry)
  std::vector<int> ls_face;              // face id of a boundary entry, else -1
  std::vector<double> ls_w;              // [n_entries][3]
  int64_t ls_degenerate = 0;

  int periodic_partner_cell(int64_t f_bnd) const {
    int pb = periodic_pair[f_bnd];
    if (pb < 0) return -1;
    return owner[n_int_faces + pb];
  }
};

// Builds connectivity, geometry, periodic pairs (patches whose bc is BC_PERIODIC) and the LS
// stencil.  Returns 0 on success, a negative code otherwise (message in *err if non-null).
int build_mesh(const RawMesh& raw, const int* patch_bc, Mesh& m, std::string* err = nullptr);

// Face-based mesh as an OpenFOAM polyMesh holds it (src/mesh/mod_foam_reader.f90:foam_read):
// every face's node list in OpenFOAM order (internal faces first, owner < neighbour, then the
// boundary faces of the patches), the owner of every face, the neighbour of every internal face,
// and each patch's face range (startFace, nFaces; absolute face indices).
struct PolyMesh {
  int64_t n_points = 0;
  const double* xyz = nullptr;           // [n_points][3]
  int64_t n_faces = 0;
  const int64_t* face_off = nullptr;     // [n_faces+1]
  const int* face_nodes = nullptr;
  const int* owner = nullptr;            // [n_faces]
  int64_t n_int_faces = 0;
  const int* neighbour = nullptr;        // [n_int_faces]
  int n_patches = 0;
  const int64_t* patch_start = nullptr;  // [n_patches] startFace
  const int64_t* patch_nfaces = nullptr; // [n_patches]
};

// The polyhedral set-up of the reference's OpenFOAM path: faces kept in the file's order, polygon
// face geometry (fan from the first node, area-weighted centre), cell centroids and volumes from
// the faces (polyhedron moments about a vertex of the cell), cell vertex lists in face order;
// then the same face metrics, periodic pairing and LS stencil as build_mesh.  Negative codes:
// -5 corrupt connectivity, -6 owner >= neighbour on an internal face, -7 patch ranges that do not
// cover the boundary faces, -8 an odd number of periodic patches.
int build_mesh_poly(const PolyMesh& pm, const int* patch_bc, Mesh& m, std::string* err = nullptr);

// Stages of build_mesh that the device builder (csrc/cuda/meshgpu.cu) shares: the cell -> face
// CSR from owner/neighbour, and the periodic pairing with its interpolation weights.
void build_cell_faces(Mesh& m);
int build_periodic(Mesh& m, std::string* err);

// Smoothstep blend of the eps.grad skewness correction (src/mesh/mod_mesh.f90:497-505).
inline double refine_blend_weight(double skew) {
  double t = (skew - SKEW_BLEND_LO) / (SKEW_BLEND_HI - SKEW_BLEND_LO);
  t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
  return 1.0 - t * t * (3.0 - 2.0 * t);
}

}  // namespace dpm
