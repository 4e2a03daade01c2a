"""The display transform on a B200: the bytes equal the reference's own kernels' bytes, bit for bit.

The reference turns an image's FP64 sums into a screen's bytes with rgba8_kernel (src/gpu/display.cu:26; the books'
gamma-2 bytes) and tone_map_kernel (src/gpu/tonemap.cu:25 with tone_curves.cuh; none, AgX and PBR Neutral, dithered),
both compiled -fmad=false (CMakeLists.txt:159-165). Those kernels, built from the reference's sources into oracle/_ref,
are run on the same sums as this library's display transform:

* synthetic sums that reach every branch (0, negatives, NaN, +-inf, huge values, the sRGB knee, the AgX middle, the
  0.999 clamp, the PBR Neutral toe and shoulder) under every tone map and several exposures;
* a rendered image (the glass Cornell box; a tone-mapped HDR view of the mesh scene under its sun) through a session's
  display(), and a served request's frame through the server's display.
"""
import numpy as np
import pytest

from oracle import ref_gpu

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_gpu.available(), reason="the reference's renderer was not built here")]

TONES = ["books", "none", "agx", "neutral"]


def _edge_sums(h=61, w=97, seed=5):
    rng = np.random.default_rng(seed)
    sums = np.concatenate([rng.exponential(1.0, size=h * w * 3 // 2),
                           10.0 ** rng.uniform(-8, 6, size=h * w * 3 - h * w * 3 // 2)])
    rng.shuffle(sums)
    special = [0.0, -0.0, -1.0, np.nan, np.inf, -np.inf, 1e300, 3.5e38, 0.0031308, 0.0031307, 0.0031309, 1.0,
               0.999 ** 2, 0.998001, (255 / 256) ** 2, 0.18, 0.08, 0.0800001, 0.76, 0.7600001, 16.29, 0.000176,
               2.0 ** -149, 5e-324]
    sums[: len(special)] = special
    return sums.reshape(h, w, 3)


def _ours_device(rt, sums, passes, tone, exposure):
    import torch

    h, w, _ = sums.shape
    d_sums = torch.tensor(sums, dtype=torch.float64, device="cuda").contiguous()
    d_rgba = torch.zeros((h, w, 4), dtype=torch.uint8, device="cuda")
    rt.display_device(d_sums.data_ptr(), w, h, passes, d_rgba.data_ptr(), tone=tone, exposure=exposure)
    torch.cuda.synchronize()
    return d_rgba.cpu().numpy()


@pytest.mark.parametrize("tone,exposure", [("books", 0.0), ("none", 0.0), ("none", 3.25), ("agx", 0.0),
                                           ("agx", -2.5), ("agx", 24.0), ("neutral", 0.0), ("neutral", 1.0),
                                           ("neutral", -24.0)])
@pytest.mark.parametrize("passes", [1, 7])
def test_device_display_equals_the_references_kernels(rt, tone, exposure, passes):
    sums = _edge_sums()
    ours = _ours_device(rt, sums, passes, tone, exposure)
    ref = ref_gpu.display_bytes(sums, 1.0 / passes, tone, exposure)
    assert ours.shape == ref.shape
    bad = np.argwhere(ours != ref)
    assert bad.size == 0, (bad[:5], [sums[tuple(b[:2])] for b in bad[:5]])
    assert np.all(ours[..., 3] == 255)


@pytest.mark.parametrize("tone", TONES)
def test_session_display_equals_the_references_kernels(rt, tone):
    s = rt.builtin_scene("glass", width=160, spp=16)
    session = rt.Session(rt.Scene(s), seed=3)
    session.render_to(48)
    exposure = 0.0 if tone == "books" else 1.5
    ours = session.display(tone, exposure)
    # pixels() is the sums times 1 / passes in double: the display kernel's own light, so scale 1 gives its bytes
    ref = ref_gpu.display_bytes(session.pixels(), 1.0, tone, exposure)
    assert np.array_equal(ours, ref)


def test_hdr_view_through_agx(rt):
    """The mesh scene's sun (radiance 5e4) under AgX: highlights roll off instead of clipping; bytes as the
    reference's."""
    s = rt.builtin_scene("mesh-ggx", width=192, spp=4, mesh_level=5, env_width=256)
    session = rt.Session(rt.Scene(s), seed=4)
    session.render_to(16)
    for tone, ev in (("agx", -3.0), ("neutral", 0.0), ("books", 0.0)):
        assert np.array_equal(session.display(tone, ev), ref_gpu.display_bytes(session.pixels(), 1.0, tone, ev))


def test_served_frame_display(rt):
    desc = rt.builtin_scene("glass", width=64, spp=16)
    scene = rt.Scene(desc)
    server = rt.Server(hbm_budget_bytes=1 << 30, step_seconds=0.005)
    rid = server.submit(scene, desc.camera, 5, 32)
    for _ in range(200):
        server.step()
        if server.poll(rid)["state"] == "done":
            break
    frame = server.display(rid, "neutral", 0.5)
    pixels = server.fetch(rid)
    assert np.array_equal(frame, ref_gpu.display_bytes(pixels, 1.0, "neutral", 0.5))
    server.close()


def test_display_refusals(rt):
    s = rt.builtin_scene("glass", width=32, spp=4)
    session = rt.Session(rt.Scene(s), seed=3)
    with pytest.raises(rt.LogicError):
        session.display()  # no complete pass yet
    session.render_to(4)
    with pytest.raises(ValueError):
        session.display("books", 1.0)
    with pytest.raises(ValueError):
        session.display("agx", 25.0)


def test_session_files(rt, oracle, tmp_path):
    """A session's PFM is its pixels as float32 (ImageCompare's input); its PNG the display's bytes; its mean
    radiance image::mean_radiance of its pixels."""
    s = rt.builtin_scene("glass", width=64, spp=16)
    session = rt.Session(rt.Scene(s), seed=8)
    session.render_to(16)
    session.save(str(tmp_path / "g.pfm"))
    px = session.pixels()
    assert np.array_equal(oracle.load_pfm(str(tmp_path / "g.pfm")), px.astype(np.float32).astype(np.float64))
    assert session.mean_radiance() == rt.mean_radiance(px)
    session.save(str(tmp_path / "g.png"), "agx", 0.0)
    from test_image_io import _decode_png  # the tests' folder is on sys.path under pytest

    assert np.array_equal(_decode_png(tmp_path / "g.png"), session.display("agx", 0.0)[..., :3])
