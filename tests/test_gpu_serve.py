"""GPU tests of the served form: requests arrive while others are on the GPU,
are admitted into batches as lanes and memory free up, and each result must
be the same, bit for bit, as the plain one-frame render of the request alone
(tolerance zero: batching changes no arithmetic)."""

import threading
import time

import numpy as np
import pytest

import gsplat_ffi as ffi
import gsplat_scenes

pytestmark = pytest.mark.gpu

SIZES = [(256, 256), (320, 200), (400, 300), (97, 61)]


def _scenes():
    rng = np.random.default_rng(5)
    a = gsplat_scenes.make_scene(rng, gsplat_scenes.gmm_means(rng, 4000), -3.5, 0.6, 0.5, 1.5, 2)
    b, _, _, _ = gsplat_scenes.config1(seed=6)
    c = gsplat_scenes.make_scene(rng, gsplat_scenes.gmm_means(rng, 30000), -4.2, 0.6, 0.5, 1.5, 3)
    return [a, b, c]


def _requests(seed, count, nscenes):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        w, h = SIZES[int(rng.integers(len(SIZES)))]
        out.append((int(rng.integers(nscenes)), gsplat_scenes.orbit_camera(rng, (3.0, 7.0)), w, h))
    return out


def _plain_images(scenes, reqs, tile=16):
    ctxs = {}
    out = []
    for sid, cam, w, h in reqs:
        key = (sid, w, h)
        if key not in ctxs:
            ctx = ffi.Context(w, h)
            ctx.set_tile_size(tile)
            ctx.load_scene(scenes[sid])
            ctxs[key] = ctx
        ctx = ctxs[key]
        ctx.set_camera(cam)
        ctx.render_frame()
        out.append((ctx.readback_rgba8().copy(), ctx.frame_counts()))
    for c in ctxs.values():
        c.close()
    return out


def _submit_poisson(srv, reqs, rate, seed, burst=16):
    """The first `burst` requests at once, the rest as a Poisson stream."""
    rng = np.random.default_rng(seed)
    ids = []
    t0 = time.perf_counter()
    t = 0.0
    for k, (sid, cam, w, h) in enumerate(reqs):
        t += 0.0 if k < burst else rng.exponential(1.0 / rate)
        delay = t0 + t - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        ids.append(srv.submit(sid, cam, w, h))
    return ids


def test_served_results_equal_alone():
    scenes = _scenes()
    reqs = _requests(1, 60, len(scenes))
    with ffi.Server(lanes=2, max_views=16) as srv:
        for s in scenes:
            srv.add_scene(s)
        ids = _submit_poisson(srv, reqs, rate=3000.0, seed=2)
        infos = [srv.wait(i) for i in ids]
        assert all(i.status == ffi.REQUEST_DONE for i in infos)
        # requests that arrived while the lanes were busy ran together
        assert max(i.batch_views for i in infos) > 1
        st = srv.stats()
        assert st.completed == len(reqs) and st.failed == 0
        assert st.batches < len(reqs)
        assert 0 < st.p50_ms <= st.p99_ms <= st.max_ms
        assert st.views_per_s > 0
        plain = _plain_images(scenes, reqs)
        for k, rid in enumerate(ids):
            img = srv.read_rgba8(rid)
            ref, counts = plain[k]
            assert np.array_equal(img, ref), f"request {k}"
            assert infos[k].visible_count == counts.visible
            assert infos[k].tile_pairs == counts.tile_keys
            srv.release(rid)


def test_served_concurrent_submitters_and_budget():
    """Four client threads submit at once; a small work budget limits how
    many requests a batch admits. Every result is still exact."""
    scenes = _scenes()
    reqs = _requests(3, 48, len(scenes))
    budget = 96 << 20
    with ffi.Server(lanes=3, max_views=64, work_budget=budget) as srv:
        for s in scenes:
            srv.add_scene(s)
        ids = [None] * len(reqs)

        def client(part):
            for k in range(part, len(reqs), 4):
                sid, cam, w, h = reqs[k]
                ids[k] = srv.submit(sid, cam, w, h)

        threads = [threading.Thread(target=client, args=(p,)) for p in range(4)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        infos = [srv.wait(i) for i in ids]
        assert all(i.status == ffi.REQUEST_DONE for i in infos)
        st = srv.stats()
        assert st.completed == len(reqs)
        assert st.peak_admitted_bytes <= budget
        plain = _plain_images(scenes, reqs)
        for k, rid in enumerate(ids):
            assert np.array_equal(srv.read_rgba8(rid), plain[k][0]), f"request {k}"


def test_served_pair_overflow_is_rerun_exactly():
    r2 = np.random.default_rng(9)
    means = r2.uniform(-2, 2, (3000, 3)).astype(np.float32)
    big = gsplat_scenes.make_scene(r2, means, -0.5, 0.3, 2.0, 0.5, 0)
    scenes = _scenes() + [big]
    reqs = _requests(4, 8, 3)
    reqs.insert(3, (3, gsplat_scenes.camera((0.0, 0.0, -3.0), (0, 0, 0), 70.0), 640, 480))
    with ffi.Server(lanes=2, max_views=8, tile=8) as srv:
        for s in scenes:
            srv.add_scene(s)
        ids = [srv.submit(*r) for r in reqs]
        infos = [srv.wait(i) for i in ids]
        assert all(i.status == ffi.REQUEST_DONE for i in infos)
        assert srv.stats().reruns >= 1
        plain = _plain_images(scenes, reqs, tile=8)
        for k, rid in enumerate(ids):
            assert np.array_equal(srv.read_rgba8(rid), plain[k][0]), f"request {k}"


def test_served_errors():
    scenes = _scenes()
    with ffi.Server(lanes=1) as srv:
        srv.add_scene(scenes[0])
        cam = gsplat_scenes.default_camera()
        with pytest.raises(ffi.GsplatError) as e:
            srv.submit(7, cam, 32, 32)
        assert e.value.code == ffi.INVALID_ARGUMENT
        with pytest.raises(ffi.GsplatError) as e:
            srv.submit(0, cam, 0, 32)
        assert e.value.code == ffi.INVALID_ARGUMENT
        with pytest.raises(ffi.GsplatError) as e:
            srv.poll(12345)
        assert e.value.code == ffi.INVALID_ARGUMENT
        rid = srv.submit(0, gsplat_scenes.camera((0, 0, -5), (0, 0, 0), 50.0), 64, 64)
        info = srv.wait(rid)
        assert info.status == ffi.REQUEST_DONE and info.latency_ms > 0
        srv.release(rid)
        with pytest.raises(ffi.GsplatError):
            srv.read_rgba8(rid)
    with pytest.raises(ffi.GsplatError) as e:
        ffi.Server(lanes=9)
    assert e.value.code == ffi.INVALID_ARGUMENT


def test_reserved_result_pool_serves_without_pinning_on_demand():
    """A server created with a pinned result reserve carves its result
    buffers from the reserved slabs: serving a stream allocates no further
    pinned memory and no launch waits on an allocation, and the results are
    still those of the plain render."""
    scenes = _scenes()
    reqs = _requests(3, 40, len(scenes))
    with ffi.Server(lanes=2, max_views=16, result_pool_mib=256) as srv:
        for s in scenes:
            srv.add_scene(s)
        ids = _submit_poisson(srv, reqs, rate=2000.0, seed=4)
        infos = [srv.wait(i) for i in ids]
        assert all(i.status == ffi.REQUEST_DONE for i in infos)
        st = srv.stats()
        assert st.pinned_slabs == 4  # 256 MiB of 64 MiB slabs, nothing more
        assert st.pinned_alloc_ms < 5.0  # carving a reserved slab, no pinning
        plain = _plain_images(scenes, reqs)
        for k, rid in enumerate(ids):
            assert np.array_equal(srv.read_rgba8(rid), plain[k][0]), f"request {k}"
            srv.release(rid)


def test_served_overload_sheds_requests_queued_past_the_bound():
    """Overload with a queueing bound: one lane, one request per batch, a
    burst far above the rate the lane serves. Requests still queued 5 ms after
    their submit are shed (FAILED, UNSUPPORTED) when the lane next takes work;
    every request that runs was admitted within the bound, and its image is
    still the plain render's."""
    scenes = _scenes()
    reqs = _requests(31, 120, len(scenes))
    plain = _plain_images(scenes, reqs)
    with ffi.Server(lanes=1, max_views=1, max_queue_ms=5) as srv:
        for s in scenes:
            srv.add_scene(s)
        ids = [srv.submit(*r) for r in reqs]
        shed = 0
        for k, rid in enumerate(ids):
            info = srv.wait(rid)
            if info.status == ffi.REQUEST_FAILED:
                assert info.error_code == ffi.UNSUPPORTED
                assert info.queue_ms > 5.0
                shed += 1
            else:
                assert info.status == ffi.REQUEST_DONE
                assert info.queue_ms <= 5.0 + 1.0, info.queue_ms
                assert np.array_equal(srv.read_rgba8(rid), plain[k][0]), k
            srv.release(rid)
        st = srv.stats()
        assert shed > 0 and st.shed == shed and st.failed >= shed
        assert st.completed + shed == len(reqs)
