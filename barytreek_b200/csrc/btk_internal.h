// Internal declarations shared by the host and device translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/barytreek_b200.h"

static_assert(sizeof(btk_run_config) == 64, "RunConfig layout (src/structs.hpp:6-22)");
static_assert(sizeof(btk_tree_info) == 16, "TreeInfo layout (src/structs.hpp:24-28)");
static_assert(sizeof(btk_panel_2d) == 80, "TreePanel_2d layout (src/structs.hpp:30-45)");
static_assert(sizeof(btk_panel_3d) == 112, "TreePanel_3d layout (src/structs.hpp:47-66)");
static_assert(offsetof(btk_panel_3d, is_leaf) == 44, "TreePanel_3d is_leaf offset");
static_assert(offsetof(btk_panel_3d, max_x) == 48, "TreePanel_3d max_x offset");
static_assert(offsetof(btk_panel_3d, min_z) == 80, "TreePanel_3d min_z offset");
static_assert(offsetof(btk_panel_3d, max_z) == 88, "TreePanel_3d max_z offset");
static_assert(offsetof(btk_panel_3d, radius) == 96, "TreePanel_3d radius offset");
static_assert(offsetof(btk_panel_3d, point_count) == 104, "TreePanel_3d point_count offset");
static_assert(offsetof(btk_panel_2d, max_x) == 32, "TreePanel_2d max_x offset");
static_assert(offsetof(btk_panel_2d, point_count) == 72, "TreePanel_2d point_count offset");
static_assert(sizeof(btk_interact_pair) == 12, "interact_pair layout (src/structs.hpp:71-75)");
static_assert(offsetof(btk_run_config, fmm_theta) == 16, "RunConfig fmm_theta offset");
static_assert(offsetof(btk_run_config, ker_eps) == 48, "RunConfig ker_eps offset");

namespace btk {

// Degree limit of the device kernels (stack/shared arrays are sized by it).
constexpr int kMaxDegree = 12;
constexpr int kMaxNodes = kMaxDegree + 1;

// Error plumbing: thread-local message + status.
btk_status set_error(btk_status s, const std::string& msg);
btk_status cuda_error(cudaError_t e, const char* what);
void count_launch(int n = 1);

#define BTK_CUDA(call)                                            \
  do {                                                            \
    cudaError_t e_ = (call);                                      \
    if (e_ != cudaSuccess) return ::btk::cuda_error(e_, #call);   \
  } while (0)
#define BTK_CHECK(cond, status, msg)                              \
  do {                                                            \
    if (!(cond)) return ::btk::set_error((status), (msg));        \
  } while (0)
#define BTK_TRY(expr)                                             \
  do {                                                            \
    btk_status s_ = (expr);                                       \
    if (s_ != BTK_OK) return s_;                                  \
  } while (0)

// Geometry of one panel in a dimension-agnostic form (device-friendly).
struct PanelGeom {
  double lo[3], hi[3];
};

// Flattened tree metadata used for planning (host) and on the device.
struct HostTree {
  int dim = 3;
  int panel_count = 0;
  int levels = 0;
  std::vector<int> level_start;  // levels+1
  std::vector<PanelGeom> geom;
  std::vector<int> parent, level, is_leaf, point_count;
  std::vector<int> child;  // panel_count * (1<<dim), -1 if none
};

void host_tree_from_panels(int dim, const void* panels, int panel_count, const int* level_start, int levels,
                           HostTree& out);
bool host_tree_from_panels_nolevels(int dim, const void* panels, int panel_count, HostTree& out);

}  // namespace btk
