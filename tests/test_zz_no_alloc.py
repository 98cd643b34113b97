"""bnxRenderStructuredNoAlloc: the entry point for callers that cannot
allocate device memory while rendering (applications that own all GPU
memory and pass this library only their own buffers, or frame loops that
must not stall on cudaMalloc's implicit synchronisation).

Through the C ABI it must give the same frames as the regular bnRender path
(bit-exact, the bar every parity test here uses), on two calls in a row that
reuse its static scratch, and reject volumes beyond its fixed scratch size.
This file is named so pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from barney_b200 import synth
from tests.helpers import assert_bitexact, small_blob_scene, small_noise_scene

pytestmark = pytest.mark.gpu

F3 = ctypes.c_float * 3


class BNXNoAllocFrame(ctypes.Structure):
    _fields_ = [("voxels", ctypes.c_void_p), ("voxelType", ctypes.c_int), ("dims", ctypes.c_int * 3),
                ("gridOrigin", F3), ("gridSpacing", F3), ("transferFunction", ctypes.c_void_p),
                ("numTFValues", ctypes.c_int), ("domain", ctypes.c_float * 2), ("densityAt1", ctypes.c_float),
                ("cameraPosition", F3), ("cameraDirection", F3), ("cameraUp", F3), ("fovy", ctypes.c_float),
                ("bgColor", ctypes.c_float * 4), ("ambientRadiance", ctypes.c_float),
                ("numDirLights", ctypes.c_int), ("dirLights", ctypes.c_void_p), ("hgPhase", ctypes.c_int),
                ("anisotropy", ctypes.c_float), ("scatteringAlbedo", ctypes.c_float),
                ("width", ctypes.c_int), ("height", ctypes.c_int), ("accumID", ctypes.c_int),
                ("pathsPerPixel", ctypes.c_int), ("accum", ctypes.c_void_p), ("color", ctypes.c_void_p),
                ("colorFormat", ctypes.c_int)]


class NoAllocCall:
    """Device buffers owned by the caller (this test), one frame description."""

    def __init__(self, d):
        import torch
        import barney_b200 as bn
        self.bn = bn
        self.vox = torch.from_numpy(np.ascontiguousarray(d["voxels"])).cuda()
        self.tf = torch.from_numpy(np.ascontiguousarray(d["tf"], np.float32)).cuda()
        self.accum = torch.zeros((d["height"], d["width"], 4), dtype=torch.float32, device="cuda")
        self.color = torch.zeros((d["height"], d["width"], 4), dtype=torch.float32, device="cuda")
        lights = d.get("dir_lights", [])
        self.lights = np.array([[*l["direction"], l.get("radiance", 1.0), *l.get("color", (1, 1, 1))]
                                for l in lights], np.float32).reshape(-1, 7)
        f = BNXNoAllocFrame()
        f.voxels = self.vox.data_ptr()
        f.voxelType = bn.VOXEL_FORMATS[d["dtype"]]
        nz, ny, nx = d["voxels"].shape
        f.dims[:] = (nx, ny, nz)
        f.gridOrigin[:] = d.get("origin", (0.0, 0.0, 0.0))
        f.gridSpacing[:] = d["spacing"]
        f.transferFunction = self.tf.data_ptr()
        f.numTFValues = self.tf.shape[0]
        f.domain[:] = d.get("domain", (0.0, 1.0))
        f.densityAt1 = d["density"]
        cam = d["camera"]
        f.cameraPosition[:] = cam["position"]
        f.cameraDirection[:] = cam["direction"]
        f.cameraUp[:] = cam.get("up", (0.0, 1.0, 0.0))
        f.fovy = cam.get("fovy", 60.0)
        f.bgColor[:] = d.get("bg_color", (0.0, 0.0, 0.0, 1.0))
        f.ambientRadiance = d.get("ambient", 1.0)
        f.numDirLights = self.lights.shape[0]
        f.dirLights = self.lights.ctypes.data if self.lights.size else None
        f.hgPhase = 1 if d.get("phase", "simple") == "hg" else 0
        f.anisotropy = d.get("anisotropy", 0.6)
        f.scatteringAlbedo = d.get("scattering_albedo", 0.9)
        f.width, f.height = d["width"], d["height"]
        f.colorFormat = bn.BN_FLOAT4
        f.accum = self.accum.data_ptr()
        f.color = self.color.data_ptr()
        self.f = f

    def render(self, accum_id, spp):
        import torch
        self.f.accumID = accum_id
        self.f.pathsPerPixel = spp
        L = self.bn.lib()
        rc = L.bnxRenderStructuredNoAlloc(ctypes.byref(self.f), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        assert rc == 0, L.bnGetLastErrorString()
        return self.color.cpu().numpy()


def regular_path(d, spp, renders):
    import barney_b200 as bn
    r = bn.VolumeRenderer(d, color_format="float4")
    try:
        r.set_spp(spp)
        out = []
        for _ in range(renders):
            r.render()
            out.append(r.read().copy())
        return out
    finally:
        r.close()


def test_no_alloc_matches_bnrender_on_two_calls_in_a_row():
    # two different volumes back to back: the second call must rebuild the
    # shared majorant scratch and clear the shared counters
    for d, spp in ((small_noise_scene(n=40, w=48, h=32), 3), (small_blob_scene(n=24, w=40, h=36), 2)):
        expect = regular_path(d, spp, renders=2)
        call = NoAllocCall(d)
        first = call.render(0, spp)            # starts the frame
        second = call.render(spp, spp)         # continues the accumulation
        assert_bitexact(first, expect[0], "first call")
        assert_bitexact(second, expect[1], "second call")


def test_no_alloc_rejects_volume_beyond_scratch():
    import barney_b200 as bn
    d = synth.scene(np.zeros((2, 1025, 16393), np.uint8), "u8", 8, 8, synth.tf_linear_ramp(16), 1.0,
                    synth.DEFAULT_CAMERA)  # 2049 x 128 x 1 macrocells > 64^3
    call = NoAllocCall(d)
    call.f.accumID, call.f.pathsPerPixel = 0, 1
    L = bn.lib()
    L.bnClearLastError()
    rc = L.bnxRenderStructuredNoAlloc(ctypes.byref(call.f), None)
    assert rc == 2
    assert b"macrocells" in L.bnGetLastErrorString()
    L.bnClearLastError()
