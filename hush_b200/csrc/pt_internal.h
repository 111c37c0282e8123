// Shared between the path tracer's host scene code (pt_scene.cu) and its kernel (pt_kernel.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "hush.h"

namespace pt {

// Device views of a built scene, in the reference's GPU layouts (see pt_scene.cu).
struct SceneView {
  const float4 *nodes;   // 4 per packed node
  const float4 *tris;    // 3 per triangle
  const uint4 *tri_idx;  // 1 per triangle
  const float4 *verts;   // 3 per vertex
  const float4 *mats;    // 5 per material
  const uint8_t *tex;    // rgba8 layers x 11 mips
  int tex_layers;
};

// The environment map: rgba16float texels and the alias table (256 x 128 cells).
struct EnvView {
  const uint2 *texels;
  int w, h;
  const float4 *table;
};

size_t tex_layer_bytes();
int fail(int code, const std::string &msg);
SceneView scene_view(const hush_pt_scene_t *s);
int scene_device(const hush_pt_scene_t *s);
bool scene_built(const hush_pt_scene_t *s);

}  // namespace pt
