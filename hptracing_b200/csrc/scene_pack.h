// Host packer: reference KD-tree + triangles -> traversal layout.
#pragma once

#include <vector>

#include "device_types.h"
#include "host.h"

namespace hpt {

struct PackedScene {
  std::vector<DevNode> nodes;
  std::vector<DevLeaf> leaves;
  std::vector<int32_t> refs;   // triangle ids in leaf order
  std::vector<DevTri> tris;    // one record per triangle
  float root_lo[3], root_hi[3];
  int max_depth = 0;
};

// The first bfs_nodes node slots are filled breadth-first from the root.
hpt_status pack_scene(const hpt_scene_desc& desc, int bfs_nodes, PackedScene& out);

}  // namespace hpt
