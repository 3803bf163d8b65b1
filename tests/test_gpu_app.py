"""GPU tests of the output utilities, the headless Application mirror and the
research_renderer.py entry point."""
import ctypes as C
import subprocess
import sys
import zlib
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


def _stream(torch):
    return torch.cuda.current_stream().cuda_stream


def tonemap_ref(hdr, exposure):
    """Application.cpp:853-866 restated in float32 numpy."""
    v = hdr[..., :3].astype(np.float32) * np.float32(exposure)
    v = (v * (np.float32(2.51) * v + np.float32(0.03))) / (v * (np.float32(2.43) * v + np.float32(0.59)) + np.float32(0.14))
    v = np.clip(v, 0, 1).astype(np.float32)
    v = np.power(v, np.float32(1.0 / 2.2)).astype(np.float32)
    out = np.empty(hdr.shape[:2] + (4,), np.uint8)
    out[..., :3] = (v * np.float32(255.0) + np.float32(0.5)).astype(np.uint8)
    out[..., 3] = 255
    return out


def test_tonemap_matches_reference_math(rr, ctx, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(2)
    hdr = (rng.random((61, 77, 4)) ** 3 * 20).astype(np.float32)
    t = torch.from_numpy(hdr).cuda()
    ldr = torch.empty((61, 77, 4), dtype=torch.uint8, device="cuda")
    ctx.check(rr.lib().rr_tonemap_execute(ctx.handle, t.data_ptr(), 77, 61, 1.3, ldr.data_ptr(), _stream(torch)))
    g = ldr.cpu().numpy().astype(int)
    ref = tonemap_ref(hdr, 1.3).astype(int)
    # powf differs from the host pow by at most an ulp, so a byte may round differently
    assert np.abs(g - ref).max() <= 1
    assert (g == ref).mean() > 0.999


def test_image_mse_fp64(rr, ctx, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(4)
    a = rng.random((50, 70, 4)).astype(np.float32)
    b = rng.random((50, 70, 4)).astype(np.float32)
    ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    ctx.check(rr.lib().rr_image_mse(ctx.handle, ta.data_ptr(), tb.data_ptr(), 70, 50, 3, 5, 64, 40, out.data_ptr(),
                                    _stream(torch)))
    d = a[5:45, 3:67, :3].astype(np.float64) - b[5:45, 3:67, :3].astype(np.float64)
    assert float(out.item()) == pytest.approx(float((d * d).mean()), rel=1e-12)
    # deterministic
    out2 = torch.zeros(1, dtype=torch.float64, device="cuda")
    ctx.check(rr.lib().rr_image_mse(ctx.handle, ta.data_ptr(), tb.data_ptr(), 70, 50, 3, 5, 64, 40, out2.data_ptr(),
                                    _stream(torch)))
    assert float(out.item()) == float(out2.item())
    assert rr.lib().rr_image_mse(ctx.handle, ta.data_ptr(), tb.data_ptr(), 70, 50, 10, 5, 64, 40, out.data_ptr(),
                                 None) == 1


def test_application_accumulates_like_oracle(rr, O, torch_cuda):
    from research_b200.passes import Application
    app = Application()
    app.initialize(48, 40)
    for _ in range(12):
        app.step()
    torch_cuda.cuda.synchronize()
    g = app.accumulate.accumulated.cpu().numpy()
    assert app.accumulate.accumulated_spp == 12
    hs = rr.HostScene.cornell(0)
    osc = O.OracleScene(hs.arrays, use_bvh=False)
    cam = rr.camera_data(rr.camera_desc(48, 40))
    imgs, _ = O.pathtrace(osc, cam, 0, 5, 12)
    acc = np.zeros((40, 48, 4), np.float32)
    for k in range(12):
        O.accumulate(np.ascontiguousarray(imgs[k]), acc, 1 if k == 0 else 0, k)
    np.testing.assert_array_equal(g.view(np.uint32), acc.view(np.uint32))
    app.set_pass_enabled("restir_di", True)
    app.set_pass_enabled("denoise", True)
    app.step()
    assert app.compute_mse() is None  # 64x64 crop does not fit a 48x40 image (Application.cpp:909)
    app.shutdown()


def test_research_renderer_cli_writes_png(tmp_path):
    out = tmp_path / "shot.png"
    r = subprocess.run([sys.executable, str(ROOT / "research_renderer.py"), "--frames", "4", "--size", "64x48",
                        "--pass", "restir_di", "--denoise", "--screenshot", str(out)], capture_output=True, text=True,
                       timeout=300, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr
    data = out.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    # decode IDAT and check the image is not black
    i = data.index(b"IDAT")
    n = int.from_bytes(data[i - 4:i], "big")
    raw = zlib.decompress(data[i + 4:i + 4 + n])
    px = np.frombuffer(raw, np.uint8).reshape(48, 1 + 64 * 4)[:, 1:].reshape(48, 64, 4)
    assert px[..., :3].mean() > 10


def test_application_gi_and_pt_modes(rr, torch_cuda):
    """restir_gi and restir_pt through the Application: PT wins over GI
    (Application.cpp:417-421), each adds indirect light to DI's direct light,
    and the displayed image follows current_display_image."""
    from research_b200.passes import Application
    torch = torch_cuda
    app = Application()
    app.initialize(64, 48)
    app.set_pass_enabled("restir_di", True)
    for _ in range(2):
        app.step()
    di = app.displayed_image().clone()
    app.set_pass_enabled("restir_gi", True)
    for _ in range(3):
        app.step()
    assert app.displayed_image() is app.restir_gi.output
    gi = app.displayed_image().clone()
    app.set_pass_enabled("restir_pt", True)
    for _ in range(3):
        app.step()
    assert app.displayed_image() is app.restir_pt.output
    pt = app.displayed_image().clone()
    torch.cuda.synchronize()
    assert torch.isfinite(gi).all() and torch.isfinite(pt).all()
    assert gi[..., :3].mean() > di[..., :3].mean() and pt[..., :3].mean() > di[..., :3].mean()
    # without DI the indirect passes still run on the G-buffer, with no direct term
    app.set_pass_enabled("restir_di", False)
    app.step()
    assert app.displayed_image() is app.restir_pt.output
    with pytest.raises(ValueError):
        app.set_pass_enabled("unknown", True)
    app.shutdown()


def test_gltf_scene_renders_bit_exact(rr, O, ctx, torch_cuda, tmp_path):
    """A generated .glb room loaded by rr_host_scene_gltf and path traced on the
    GPU equals the oracle's render of the same arrays."""
    import gltf_files
    torch = torch_cuda
    path = str(tmp_path / "room.glb")
    gltf_files.room_scene().save(path, "glb")
    hs = rr.HostScene.gltf(path)
    scene = rr.Scene(ctx, hs.arrays)
    osc = O.OracleScene(hs.arrays, use_bvh=False)
    cam = rr.camera_data(rr.camera_desc(40, 32, eye=(0.0, 0.0, 2.9), center=(0.0, 0.0, 0.0)))
    out = torch.zeros((2, 32, 40, 4), device="cuda")
    p = rr.PtParams(3, 6, 2, 0)
    ctx.check(rr.lib().rr_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p), out.data_ptr(),
                                             _stream(torch)))
    torch.cuda.synchronize()
    o, _ = O.pathtrace(osc, cam, 3, 6, 2)
    g = out.cpu().numpy()
    np.testing.assert_array_equal(g.view(np.uint32), o.view(np.uint32))
    assert g[..., :3].mean() > 0.01
    scene.close()
    hs.close()


def test_research_renderer_cli_gltf_and_pt(tmp_path):
    import gltf_files
    scene = tmp_path / "room.gltf"
    gltf_files.room_scene().save(str(scene))
    out = tmp_path / "pt.png"
    r = subprocess.run([sys.executable, str(ROOT / "research_renderer.py"), str(scene), "--frames", "3", "--size",
                        "64x48", "--pass", "restir_di", "--pass", "restir_pt", "--screenshot", str(out)],
                       capture_output=True, text=True, timeout=300, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr
    assert "scene=room.gltf" in r.stdout and out.read_bytes()[:8] == b"\x89PNG\r\n\x1a\n"
