// Device builder of the mesh and the static operator data (setup_gpu.cu).  It produces the same
// Mesh and StaticOps, value for value, as the host builder (csrc/host/mesh.cpp, ops.cpp): every
// per-cell and per-face quantity is computed on the GPU in the host builder's operation order
// (the translation unit is compiled without floating-point contraction), and the work that is
// per patch or per boundary face only (periodic pairing, outlet rows) stays on the host.  The one
// exception is the SGS filter tensor, whose scale takes a cube root by pow(); device and host
// pow may round differently in the last place.
#pragma once
#include <string>
#include <vector>

#include "../../../include/dopamine_b200.h"
#include "../host/mesh.hpp"
#include "../host/ops.hpp"

namespace dpm {

// Wall-clock milliseconds of the set-up stages.
struct SetupTimes {
  double mesh_ms = 0.0;  // connectivity, geometry, periodic pairs, LS stencil
  double ops_ms = 0.0;   // static operators
  // device builder: raw upload, cells and face matching, faces and cell->face lists, periodic
  // pairing (host), LS stencil, static operators, download
  double stage_ms[7] = {0, 0, 0, 0, 0, 0, 0};
};

// Device-resident output of the device builder, in the layouts the time step reads (the Dev view
// of common.cuh): cell vectors [k][nc], face vectors [k][nf], ELL lists [slot][nc], pressure-
// solver face vectors [k][nfp].  The arrays are owned here until release() hands them over.
struct SetupDeviceArrays {
  double *vol = nullptr, *ivol = nullptr, *cen = nullptr, *Tinv = nullptr, *G = nullptr, *ls_w = nullptr;
  double *sf = nullptr, *nrm = nullptr, *fcen = nullptr, *eps = nullptr, *area = nullptr, *gc = nullptr;
  double *wbl = nullptr, *dcf = nullptr, *psc = nullptr, *psgcf = nullptr, *psgcw = nullptr, *psk = nullptr;
  double *pskrc = nullptr, *Aval = nullptr, *Adinv = nullptr;
  int *cf = nullptr, *cps = nullptr, *cbn = nullptr, *ls_idx = nullptr, *fo = nullptr, *fn = nullptr;
  int *pso = nullptr, *psn = nullptr, *psf = nullptr, *Acol = nullptr;
  std::vector<int> bps, bcanon;  // host: pressure-solver index of each periodic boundary face, canonical side
  std::vector<void*> owned;
  std::vector<void*> release() {
    std::vector<void*> v;
    v.swap(owned);
    return v;
  }
  ~SetupDeviceArrays();
};

// Status of the device builder when a mesh is beyond its per-cell capacities (more than 64 vertices
// or 16 faces in a cell, more than 2^31 element faces); the host builder has no such limits.
constexpr int SETUP_DEVICE_LIMIT = -100;

// Builds m and S on device `device`.  Returns 0, a negative mesh code of build_mesh (message in
// *err), or a DPM_ERR_* code from the static-operator stage / the CUDA runtime.
// dev == nullptr: every array of m and S is copied to the host (as the host builder fills them).
// Otherwise the arrays the time step reads stay in HBM (*dev), and m and S get on the host only
// what host code reads after set-up: cell centroids and volumes, owner / patch / area / centre /
// normal / d_cf of every face (boundary faces are what the host uses), the periodic pairing, the
// boundary-face operator data, the outlet rows, the switches, and the assembled matrix (the
// pressure-solver hierarchies are built on the host).
int build_setup_device(const RawMesh& raw, const dpm_patch_cfg_t* pc, const dpm_params_t& P, int device, Mesh& m,
                       StaticOps& S, std::string* err, SetupTimes* t, SetupDeviceArrays* dev = nullptr);

// The same for a face-based (OpenFOAM) mesh: the reference's polyhedral geometry
// (build_mesh_poly's checks, polygon faces, polyhedron moments, face-ordered cell vertices) on
// the device in the host builder's operation order, then the shared stages.
int build_setup_device_poly(const PolyMesh& pm, const dpm_patch_cfg_t* pc, const dpm_params_t& P, int device,
                            Mesh& m, StaticOps& S, std::string* err, SetupTimes* t, SetupDeviceArrays* dev = nullptr);

}  // namespace dpm
