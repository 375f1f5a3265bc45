// zdx_host.h -- host-side helpers shared by the C ABI, the scene loader and the zdem_gpu program.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace zdx {

// load_stl, src/main.cpp:308-371.  9 doubles per triangle.
bool stl_read(const std::string& path, std::vector<double>& tris);
// build_mesh, src/main.cpp:445-497.  props: volume, center3, radius, mean_edge, bbox_diag, inertia9, nvert.
void mesh_build(const double* tris, int64_t ntri, bool center_mesh, double* tris_out, double* props);

}  // namespace zdx
