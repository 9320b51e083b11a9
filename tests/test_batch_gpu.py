"""Dynamic studies (hrrt_batch_* through the C ABI) and the projector launch
shapes.

Every frame of a batch is bit-identical to the single-frame reconstruction of
the same inputs (hrrt_upload_inputs + hrrt_sensitivity + hrrt_init_image +
hrrt_osem(iterations) + hrrt_get_image), with uneven iteration counts, the
three storage types (f32, bf16 and fp16 terms) and both back projectors; its FP64 image sum equals
hrrt_osem's.  Every launch shape, and the autotuner's pick, gives
bit-identical images (the shape only regroups planes among threads)."""
import numpy as np
import pytest

from geoms import ALL, product_geom
from golden import inputs as I

pytestmark = pytest.mark.gpu


def frame_inputs(shape, nframes, seed):
    """Per-frame prompts (Poisson, count level varying 30x between frames),
    randoms and scatter scaled with the frame's counts."""
    rng = np.random.default_rng(seed)
    P, V, N = shape
    base = np.abs(np.sin(np.arange(N) * 0.07))[None, None, :] + 0.2
    out = []
    for f in range(nframes):
        level = float(np.exp(rng.uniform(np.log(0.2), np.log(6.0))))
        prompts = rng.poisson(level * base, size=shape).astype(np.int16)
        randoms = np.full(shape, 0.2 * level, np.float32)
        scatter = (0.1 * level * base * np.ones(shape)).astype(np.float32)
        out.append((prompts, randoms, scatter))
    return out


def single_frame(d, norm, atten, prompts, randoms, scatter, iterations, storage, bp):
    import hrrt_reconstruction_b200 as H
    with H.Context(product_geom(d)) as ctx:
        ctx.set_backprojector(bp)
        ctx.upload_inputs(prompts, randoms, norm, atten, scatter, storage=storage)
        ctx.sensitivity()
        ctx.init_image()
        st = ctx.osem(iterations)
        return ctx.get_image(), st.sum_image


@pytest.mark.parametrize("name,storage,bp", [("small3", 0, 0), ("small9", 1, 0), ("small9", 2, 0), ("small9", 0, 1)])
def test_frames_match_single_frame(name, storage, bp):
    import hrrt_reconstruction_b200 as H
    d = ALL[name]
    with H.Context(product_geom(d)) as ctx:
        shape = ctx.sino_shape
        _, _, norm, atten, _ = I.sinograms(*shape)
        iters = [2, 1, 3, 1]
        frames = frame_inputs(shape, len(iters), seed=31 + storage + 2 * bp)
        ctx.set_backprojector(bp)
        with ctx.batch(len(iters), norm=norm, atten=atten, storage=storage) as b:
            for f, (p, r, s) in enumerate(frames):
                b.set_frame(f, p, r, s, iterations=iters[f])
            st = b.run()
            got = [b.get_image(f) for f in range(len(iters))]
            # one group; active frames per iteration 4, 2, 1: three graphs, three replays
            assert st.groups == 1 and st.graphs == 3 and st.graph_launches == 3, st.as_dict()
            assert st.subset_iterations == 16 * sum(iters)
            assert st.kernel_launches == 3 * (3 * 16 + 2)
            # a second run starts again from the uniform image and reuses the graphs
            st2 = b.run()
            assert st2.graphs == 0 and st2.graph_launches == 3
            for f in range(len(iters)):
                img, sm = b.get_image(f)
                assert np.array_equal(img.view(np.uint32), got[f][0].view(np.uint32))
                assert sm == got[f][1]
    for f, (p, r, s) in enumerate(frames):
        want, want_sum = single_frame(d, norm, atten, p, r, s, iters[f], storage, bp)
        assert np.array_equal(got[f][0].view(np.uint32), want.view(np.uint32)), f
        assert got[f][1] == want_sum, (f, got[f][1], want_sum)


def test_hrrt9_frames_match_single_frame():
    """Full-size span 9, two frames, 16-bit storage."""
    import hrrt_reconstruction_b200 as H
    d = ALL["hrrt9"]
    with H.Context(product_geom(d)) as ctx:
        shape = ctx.sino_shape
        _, _, norm, atten, _ = I.sinograms(*shape)
        frames = frame_inputs(shape, 2, seed=41)
        with ctx.batch(2, norm=norm, atten=atten, storage=H.STORE_16) as b:
            for f, (p, r, s) in enumerate(frames):
                b.set_frame(f, p, r, s, iterations=1 + f)
            st = b.run()
            assert st.subset_iterations == 16 * 3
            got = [b.get_image(f) for f in range(2)]
    for f, (p, r, s) in enumerate(frames):
        want, want_sum = single_frame(d, norm, atten, p, r, s, 1 + f, H.STORE_16, 0)
        assert np.array_equal(got[f][0].view(np.uint32), want.view(np.uint32)), f
        assert got[f][1] == want_sum


def test_batch_state_errors():
    import hrrt_reconstruction_b200 as H
    d = ALL["small9"]
    with H.Context(product_geom(d)) as ctx:
        shape = ctx.sino_shape
        prompts, randoms, norm, atten, scatter = I.sinograms(*shape)
        b = ctx.batch(2, norm=norm, atten=atten)
        with pytest.raises(H.HrrtError):
            b.set_frame(2, prompts, randoms)
        with pytest.raises(H.HrrtError):
            b.set_frame(0, prompts, randoms, iterations=0)
        b.set_frame(0, prompts, randoms, scatter)
        with pytest.raises(H.HrrtError):
            b.run()  # frame 1 missing
        with pytest.raises(H.HrrtError):
            ctx.upload_inputs(prompts, randoms, norm, atten, scatter)  # the batch owns the inputs
        with pytest.raises(H.HrrtError):
            ctx.batch(1)  # one batch per context
        b.close()
        ctx.upload_inputs(prompts, randoms, norm, atten, scatter)
        ctx.sensitivity()


def _shapes(ctx):
    import hrrt_reconstruction_b200 as H
    out = []
    for pl in (7, 9, 11):
        for pw in (0, 2, 3, 4, 6):
            for kb in (4, 8):
                for nt in (0, 256, 384):
                    try:
                        ctx.set_tuning(pl, pw, kb, nt)
                    except H.HrrtError:
                        continue
                    out.append((pl, pw, kb, nt, 0))
    # the back projector's tile width (tasks side by side along the planes)
    for kb, nt in ((8, 0), (4, 256)):
        for r in (1, 2, 4, 8, 16, 32):
            out.append((9, 0, kb, nt, r))
    with pytest.raises(H.HrrtError):
        ctx.set_tuning(9, 0, 8, 0, 3)
    ctx.set_tuning()
    return out


@pytest.mark.parametrize("name", ["small3", "hrrt9"])
def test_launch_shapes_bit_identical(name):
    import hrrt_reconstruction_b200 as H
    from oracle.oracle import Oracle
    d = ALL[name]
    with H.Context(product_geom(d)) as ctx:
        shape = ctx.sino_shape
        prompts, randoms, norm, atten, scatter = I.sinograms(*shape)
        ctx.upload_inputs(prompts, randoms, norm, atten, scatter)
        ctx.sensitivity()
        ctx.init_image()
        ctx.osem_subsets(0, 1)
        img0 = ctx.get_image_xyz()
        shapes = _shapes(ctx)
        assert (9, 0, 8, 0, 0) in shapes and len(shapes) >= 32, shapes
        want = None
        for t in shapes:
            ctx.set_tuning(*t)
            ctx.set_image_xyz(img0)
            ctx.osem_subsets(1, 2)
            got = ctx.get_image_xyz()
            if want is None:
                want = got
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), t
        # the tuner picks one of them and leaves the image alone
        ctx.set_image_xyz(img0)
        t = ctx.autotune(repeats=2)
        assert (t.fp_planes, t.bp_planes) in {(s[0], s[2]) for s in shapes} and t.fp_ms > 0 and t.bp_ms > 0
        assert np.array_equal(ctx.get_image_xyz().view(np.uint32), img0.view(np.uint32))
        got = ctx.get_tuning()
        assert (got.fp_planes, got.fp_producer_warps, got.bp_planes) == (t.fp_planes, t.fp_producer_warps,
                                                                          t.bp_planes)
        ctx.osem_subsets(1, 2)
        assert np.array_equal(ctx.get_image_xyz().view(np.uint32), want.view(np.uint32))
    # the FP of one pair with a non-default shape still matches the oracle bit for bit
    O = Oracle(precision="f32", **d)
    with H.Context(product_geom(d)) as ctx:
        from geoms import random_image
        x = random_image(ctx.image_shape, O.cylwiny(), seed=5, zvalid=O.nz)
        ctx.set_tuning(7, 2, 4, 384)
        assert np.array_equal(ctx.fp_pair(x, 3).view(np.uint32), O.fp_pair(x, 3).view(np.uint32))


def test_batch_autotune():
    import hrrt_reconstruction_b200 as H
    d = ALL["small9"]
    with H.Context(product_geom(d)) as ctx:
        shape = ctx.sino_shape
        _, _, norm, atten, _ = I.sinograms(*shape)
        frames = frame_inputs(shape, 3, seed=51)
        with ctx.batch(3, norm=norm, atten=atten, storage=H.STORE_16) as b:
            for f, (p, r, s) in enumerate(frames):
                b.set_frame(f, p, r, s, iterations=2)
            b.run()
            want = [b.get_image(f)[0] for f in range(3)]
            t = b.autotune(repeats=2)
            assert t.fp_ms > 0
            st = b.run()
            assert st.graphs >= 1  # the new shape invalidated the captured graphs
            for f in range(3):
                assert np.array_equal(b.get_image(f)[0].view(np.uint32), want[f].view(np.uint32))
