// Device builder of the mesh and the static operator data (setup_gpu.cu).  It produces the same
// Mesh and StaticOps, value for value, as the host builder (csrc/host/mesh.cpp, ops.cpp): every
// per-cell and per-face quantity is computed on the GPU in the host builder's operation order
// (the translation unit is compiled without floating-point contraction), and the work that is
// per patch or per boundary face only (periodic pairing, outlet rows) stays on the host.  The one
// exception is the SGS filter tensor, whose scale takes a cube root by pow(); device and host
// pow may round differently in the last place.
#pragma once
#include <string>

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

// Builds m and S on device `device`.  Returns 0, a negative mesh code of build_mesh (message in
// *err), or a DPM_ERR_* code from the static-operator stage / the CUDA runtime.
int build_setup_device(const RawMesh& raw, const dpm_patch_cfg_t* pc, const dpm_params_t& P, int device, Mesh& m,
                       StaticOps& S, std::string* err, SetupTimes* t);

}  // namespace dpm
