"""bnxRenderStructuredNoAlloc: the entry point for callers that cannot
allocate device memory while rendering (applications that own all GPU
memory and pass this library only their own buffers, or frame loops that
must not stall on cudaMalloc's implicit synchronisation).

Through the C ABI it must give the same frames as the regular bnRender path
(bit-exact, the bar every parity test here uses), on two calls in a row that
reuse its static scratch, for every voxel type and colour format; allocate
nothing (an allocation made to fail succeeds it no harm, and the device's
free memory does not move); accept exactly the largest grid its scratch
holds (513^3 scalars, 64^3 macrocells) and reject the next larger one.
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

    def __init__(self, d, color_format="float4"):
        import torch
        import barney_b200 as bn
        self.bn = bn
        v = d["voxels"]
        self.vox = v if isinstance(v, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(v)).cuda()
        self.tf = torch.from_numpy(np.ascontiguousarray(d["tf"], np.float32)).cuda()
        self.accum = torch.zeros((d["height"], d["width"], 4), dtype=torch.float32, device="cuda")
        if color_format == "float4":
            self.color = torch.zeros((d["height"], d["width"], 4), dtype=torch.float32, device="cuda")
        else:  # 8-bit RGBA packed in 32 bits
            self.color = torch.zeros((d["height"], d["width"]), dtype=torch.int32, device="cuda")
        self.color_format = color_format
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
        f.colorFormat = bn.COLOR_FORMATS[color_format]
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
        out = self.color.cpu().numpy()
        return out if self.color_format == "float4" else out.view(np.uint32)


def regular_path(d, spp, renders, color_format="float4"):
    import barney_b200 as bn
    r = bn.VolumeRenderer(d, color_format=color_format)
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


@pytest.mark.parametrize("dtype,color_format", [("u8", "rgba8"), ("f16", "float4"), ("f32", "rgba8_srgb")])
def test_no_alloc_voxel_types_and_colour_formats(dtype, color_format):
    d = small_noise_scene(n=33, w=40, h=24, dtype=dtype)
    expect = regular_path(d, 2, renders=2, color_format=color_format)
    call = NoAllocCall(d, color_format)
    assert_bitexact(call.render(0, 2), expect[0], f"{dtype} {color_format}: first call")
    assert_bitexact(call.render(2, 2), expect[1], f"{dtype} {color_format}: second call")


def test_no_alloc_allocates_nothing():
    """The library's own device allocations go through one wrapper; armed to
    fail the next one, a no-allocation call still succeeds (and leaves the
    failure armed for the next allocation).  The device's free memory is the
    same before and after a call."""
    import torch
    import barney_b200 as bn
    L = bn.lib()
    d = small_noise_scene(n=40, w=48, h=32)
    expect = regular_path(d, 3, renders=1)
    call = NoAllocCall(d)
    call.render(0, 3)  # warm-up: loads the kernels and looks the scratch up
    free0, _ = torch.cuda.mem_get_info()
    L.bnxInjectAllocationFailure(0)
    try:
        frame = call.render(0, 3)
        free1, _ = torch.cuda.mem_get_info()
        # the armed failure is still pending: the next library allocation fails
        with pytest.raises(bn.BarneyError):
            bn.VolumeRenderer(d)
    finally:
        L.bnxInjectAllocationFailure(-1)
        L.bnClearLastError()
    assert_bitexact(frame, expect[0], "frame with an allocation made to fail")
    assert free1 == free0, (free0, free1)


def test_no_alloc_accepts_its_largest_grid_and_rejects_the_next():
    """513^3 scalars are exactly 64^3 macrocells: accepted, and equal to
    bnRender; one more scalar along x needs 65 x 64 x 64: rejected."""
    import torch
    import barney_b200 as bn
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    vol = torch.randint(0, 256, (513, 513, 513), dtype=torch.uint8, device="cuda", generator=g)
    d = synth.scene(vol, "u8", 24, 16, synth.tf_knots(256, 1), 20.0, synth.DEFAULT_CAMERA)
    expect = regular_path(d, 1, renders=1)
    call = NoAllocCall(d)
    assert_bitexact(call.render(0, 1), expect[0], "513^3 grid")
    del call
    big = synth.scene(torch.zeros((513, 513, 514), dtype=torch.uint8, device="cuda"), "u8", 8, 8,
                      synth.tf_knots(256, 1), 20.0, synth.DEFAULT_CAMERA)
    call = NoAllocCall(big)
    call.f.accumID, call.f.pathsPerPixel = 0, 1
    L = bn.lib()
    L.bnClearLastError()
    assert L.bnxRenderStructuredNoAlloc(ctypes.byref(call.f), None) == 2
    assert b"macrocells" in L.bnGetLastErrorString()
    L.bnClearLastError()
