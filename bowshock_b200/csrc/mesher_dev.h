// Host interface of the device mesher (mesher_dev.cu, its own translation unit): grid sizes of a mesh request and the
// batched meshing on the device.
#pragma once
#include <cstdint>
#include <string>

#include "../../include/bowshock_b200.h"

namespace bkmesh {

struct Dims {
  long long ni = 0, nj = 0, i_end = 0, j_end = 0, j_sting = 0;  // the solid block (zero for a sting grid)
};

// Cell counts and block of request q after the host mesher's argument checks; false (and err) if it would refuse it.
bool dims(const bowshock_mesh_request& q, Dims& d, std::string& err);

// Nodes (x, r; case k at the sum of (ni+1)(nj+1) of the cases before it) and, when metrics is not null, the metrics
// (BOWSHOCK_MESH_METRIC_WORDS per case, same order) of n requests, built on the device and copied to the host buffers.
int mesh_batch(uint64_t n, const bowshock_mesh_request* q, int device, double* x, double* r, double* metrics, double* device_ms, std::string& err);

}  // namespace bkmesh
