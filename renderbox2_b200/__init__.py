"""renderbox2_b200: a B200 (sm_100a) ray-query and light-transport engine that
drops in for renderbox2's SBVH build -> Compact2 layout -> traversal ->
integrator path.  All compute runs in librb2.so (C++ host + CUDA kernels);
this package is a thin ctypes layer over its C ABI (include/rb2*.h)."""
from ._native import Rb2Error, lib
from .accel import (BVH, MODE_ANY, MODE_CLOSEST, MODE_OCCLUSION, NODE_ORDER_BFS, NODE_ORDER_CW8, NODE_ORDER_DFS, NODE_ORDER_WIDE4, BuildParams, CudaBvh, CudaTracer, HostPipeline,
                    Platform, Scene, TraceBatch, hits_view)
from .scenefile import SceneFile, load_scene_file
from .scenes import PerspectiveCamera, RoomScene, heightfield_for_triangles, heightfield_scene, pcg32, surface_rays

__all__ = [
    "Rb2Error", "lib", "BVH", "BuildParams", "CudaBvh", "CudaTracer", "Platform", "Scene", "hits_view", "TraceBatch",
    "HostPipeline", "MODE_CLOSEST", "MODE_ANY", "MODE_OCCLUSION", "NODE_ORDER_DFS", "NODE_ORDER_BFS", "NODE_ORDER_WIDE4", "NODE_ORDER_CW8",
    "SceneFile", "load_scene_file", "PerspectiveCamera", "RoomScene", "heightfield_for_triangles", "heightfield_scene", "pcg32", "surface_rays",
]
