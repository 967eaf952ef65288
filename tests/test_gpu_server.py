"""Serving loop with continuous batching (bielcc_server_*): results of
requests submitted at any time match the oracle; a request's result is
bit-identical alone and inside a mix of other requests; requests that arrive
while a large batch runs are admitted on another slot and finish first;
HBM-budget admission, cancellation and argument errors are host-side."""
import time

import numpy as np
import pytest

import oracle
from bielcc_b200 import abi, gpu
from bielcc_b200 import workloads as W
from conftest import TOL_FP64, TOL_MIXED, rel_l2

pytestmark = pytest.mark.gpu


def _specs(gctx, seed):
    rng = np.random.default_rng(seed)
    meshes = [W.uv_sphere(6, 12), W.perturbed_icosphere(1, seed=4), W.torus(18, 6), W.spheroid(5, 10, 1.0, 2.5)]
    out = []
    for i, cells in enumerate(meshes):
        k = [2.0, 5.0, complex(3.0, 0.2), 9.0][i]
        S = [1, 5, 3, 7][i]
        ext = float(np.max(np.linalg.norm(cells.reshape(-1, 3), axis=1)))
        pts = np.concatenate([W.shell_points(40 + 13 * i, 1.6 * ext, 3 * ext, rng),
                              W.near_points(cells, 6, 0.02, 0.2, rng)])
        out.append(dict(mesh=gctx.mesh(cells), cells=cells, J=W.po_currents(cells, abs(k), directions=S, seed=i),
                        pts=pts, k=k, mult=complex(1.0, 0.5 * i)))
    return out


def _submit(sv, sp, out_c64=True):
    return sv.submit_field(sp["mesh"], sp["J"], sp["pts"], sp["k"], mult=sp["mult"], out_c64=out_c64)


@pytest.mark.parametrize("precision,tol", [("fp64", TOL_FP64), ("mixed", TOL_MIXED)])
def test_server_results_match_oracle(gctx, precision, tol):
    specs = _specs(gctx, 1)
    sv = gpu.Server(gctx, n_slots=2, precision=precision)
    try:
        tickets = [_submit(sv, sp, out_c64=False) for sp in specs]
        for sp, t in zip(specs, tickets):
            st, lat, out = sv.wait(t)
            assert st == 0 and lat > 0
            Eo, Ho = oracle.field_EH(sp["cells"], sp["J"], sp["k"], sp["pts"], mult=sp["mult"])
            assert rel_l2(out["E"], Eo) < tol and rel_l2(out["H"], Ho) < tol
        s = sv.stats()
        assert s["completed"] == len(specs) and s["failed"] == 0 and s["bytes_reserved"] == 0
    finally:
        sv.close()


@pytest.mark.parametrize("precision,tol", [("fp64", TOL_FP64), ("mixed", TOL_MIXED)])
def test_server_adaptive_p_max2(gctx, precision, tol):
    """A server with p_max = 2: served batches run the batched kernel's far pass
    at 2 n_start (the pass the reference's loop returns) and the full schedule
    for near pairs; results against the oracle's loop. A served assembly request
    equals the direct call with the same parameters. p_max = 3 needs the
    convergence-test marks, which the batched kernel does not read: refused."""
    specs = _specs(gctx, 5)[:3]
    npm = abi.NumParam.default(n_start=4, n_start_seg=5, p_max=2, p_max_seg=2)
    sv = gpu.Server(gctx, n_slots=2, numparam=npm, precision=precision)
    try:
        tickets = [_submit(sv, sp, out_c64=False) for sp in specs]
        c64 = precision == "mixed"
        ta = sv.submit_assemble(specs[1]["mesh"], 4.0, layout="tau2", out_c64=c64)
        for sp, t in zip(specs, tickets):
            st, _, out = sv.wait(t)
            assert st == 0
            Eo, Ho = oracle.field_EH(sp["cells"], sp["J"], sp["k"], sp["pts"], npm, mult=sp["mult"])
            assert rel_l2(out["E"], Eo) < tol and rel_l2(out["H"], Ho) < tol
        st, _, out = sv.wait(ta)
        assert st == 0
        A_direct, _ = gctx.assemble_K(specs[1]["mesh"], 4.0, numparam=npm, layout=abi.LAYOUT_TAU2, c64=c64,
                                      precision=precision)
        assert np.array_equal(out["A"], A_direct)
    finally:
        sv.close()
    with pytest.raises(gpu.BielccError):
        gpu.Server(gctx, n_slots=1, numparam=abi.NumParam.default(p_max=3), precision=precision)


def test_server_request_alone_equals_in_mix(gctx):
    specs = _specs(gctx, 2)
    sv = gpu.Server(gctx, n_slots=3, precision="mixed")
    try:
        alone = {}
        for i in (0, 2, 3):
            st, _, alone[i] = sv.wait(_submit(sv, specs[i]))
            assert st == 0
        # a burst released at once: the field requests between assembly
        # requests run as shared batches on several slots
        sv.pause(True)
        tickets = []
        for rep in range(3):
            for i, sp in enumerate(specs):
                tickets.append((i, _submit(sv, sp)))
            tickets.append((-1, sv.submit_assemble(specs[1]["mesh"], 4.0)))
        sv.pause(False)
        for i, t in tickets:
            st, _, out = sv.wait(t)
            assert st == 0
            if i in alone:
                assert np.array_equal(out["E"], alone[i]["E"]) and np.array_equal(out["H"], alone[i]["H"])
        s = sv.stats()
        assert s["max_batch"] >= len(specs) and s["batches"] < s["completed"]
    finally:
        sv.close()


def test_server_small_requests_overtake_a_large_batch(gctx):
    big_cells = W.uv_sphere(64, 128)
    big = dict(mesh=gctx.mesh(big_cells), J=W.po_currents(big_cells, 2 * np.pi), k=2 * np.pi, mult=1.0,
               pts=W.shell_points(20000, 2.0, 5.0, np.random.default_rng(0)))
    small = _specs(gctx, 3)[0]
    sv = gpu.Server(gctx, n_slots=2, precision="mixed")
    try:
        tb = _submit(sv, big)
        t0 = time.monotonic()
        while sv.stats()["running"] < 1:  # the server has admitted the large request into a slot
            assert time.monotonic() - t0 < 60.0
            time.sleep(0.0002)
        ts = [_submit(sv, small) for _ in range(4)]
        lat_small = [sv.wait(t)[1] for t in ts]
        st, lat_big, _ = sv.wait(tb)
        assert st == 0
        assert max(lat_small) < lat_big
        assert sv.stats()["priority_batches"] >= 1
    finally:
        sv.close()


def test_server_cap_runs_a_large_request_alone(gctx):
    """With a cap on a batch's pairs, a request above a quarter of the cap runs
    in a batch of its own, and the small requests queued behind it go ahead
    together on the other slot; each result is the same as alone."""
    big_cells = W.uv_sphere(64, 128)
    big = dict(mesh=gctx.mesh(big_cells), J=W.po_currents(big_cells, 2 * np.pi), k=2 * np.pi, mult=1.0,
               pts=W.shell_points(20000, 2.0, 5.0, np.random.default_rng(0)))
    small = _specs(gctx, 4)
    sv = gpu.Server(gctx, n_slots=2, precision="mixed", max_batch_pairs=2 * 10**8)  # "large": > 5e7 pairs
    try:
        alone = [sv.wait(_submit(sv, sp))[2] for sp in small]
        s0 = sv.stats()
        sv.pause(True)
        tb = _submit(sv, big)  # 1.6e8 pairs, first in line
        ts = [_submit(sv, sp) for sp in small]
        sv.pause(False)
        res = [sv.wait(t) for t in ts]
        st, lat_big, _ = sv.wait(tb)
        assert st == 0 and all(r[0] == 0 for r in res)
        for (_, _, out), a in zip(res, alone):
            assert np.array_equal(out["E"], a["E"]) and np.array_equal(out["H"], a["H"])
        s = sv.stats()
        assert s["batches"] - s0["batches"] == 2 and s["max_batch"] == len(small)
        assert max(r[1] for r in res) < lat_big
        # the server's batch trace: the last two batches are the large request alone and the small ones
        tr = sv.trace()[-2:]
        assert sorted(b["n_requests"] for b in tr) == [1, len(small)]
        assert {b["slot"] for b in tr} == {0, 1}
        for b in tr:
            assert 0 <= b["admit_ms"] <= b["stage1_ms"] <= b["done_ms"] <= b["complete_ms"]
        big_b = next(b for b in tr if b["n_requests"] == 1)
        assert big_b["pairs"] == len(big["pts"]) * len(big_cells) and big_b["assembly"] == 0
    finally:
        sv.close()


def test_server_priority_settings(gctx):
    """Without overtaking, no batch takes the high-priority stream unless it is
    within the priority threshold; results do not depend on the stream."""
    specs = _specs(gctx, 5)
    outs = {}
    for overtake, prio in ((False, 0), (False, 10**9), (True, 0)):
        sv = gpu.Server(gctx, n_slots=2, precision="mixed", overtake=overtake, priority_pairs=prio)
        try:
            res = [sv.wait(_submit(sv, sp)) for sp in specs]
            assert all(r[0] == 0 for r in res)
            s = sv.stats()
            if not overtake:
                assert s["priority_batches"] == (s["batches"] if prio else 0)
            outs[(overtake, prio)] = [r[2] for r in res]
        finally:
            sv.close()
    ref = outs[(False, 0)]
    for k, v in outs.items():
        for a, b in zip(v, ref):
            assert np.array_equal(a["E"], b["E"]) and np.array_equal(a["H"], b["H"]), k


def test_server_assembly_and_resident_currents(gctx):
    torch = pytest.importorskip("torch")
    specs = _specs(gctx, 4)
    sv = gpu.Server(gctx, n_slots=2, precision="mixed")
    try:
        sp = specs[1]
        A_direct, _ = gctx.assemble_K(sp["mesh"], 4.0, layout=abi.LAYOUT_TAU2, c64=True, precision="mixed")
        st, _, out = sv.wait(sv.submit_assemble(sp["mesh"], 4.0, layout="tau2", out_c64=True))
        assert st == 0 and np.array_equal(out["A"], A_direct)
        # currents resident on the device give the same result as host currents
        Jd = torch.from_numpy(np.ascontiguousarray(sp["J"])).to("cuda:0")
        torch.cuda.synchronize()
        st1, _, o1 = sv.wait(_submit(sv, sp))
        st2, _, o2 = sv.wait(sv.submit_field(sp["mesh"], None, sp["pts"], sp["k"], mult=sp["mult"],
                                             J_dev=Jd.data_ptr(), n_rhs=sp["J"].shape[0]))
        assert st1 == st2 == 0 and np.array_equal(o1["E"], o2["E"]) and np.array_equal(o1["H"], o2["H"])
    finally:
        sv.close()


def test_server_budget_cancel_and_errors(gctx):
    specs = _specs(gctx, 5)
    sp = specs[3]
    sv = gpu.Server(gctx, hbm_budget=4 << 20, n_slots=2, precision="mixed")
    try:
        # a request larger than the whole budget is refused at submission
        many = W.shell_points(200000, 2.0, 3.0, np.random.default_rng(1))
        with pytest.raises(gpu.BielccError) as e:
            sv.submit_field(sp["mesh"], sp["J"], many, sp["k"])
        assert e.value.code == abi.ERR_BUSY
        # unknown mesh
        bad = gpu.Mesh.__new__(gpu.Mesh)
        bad.id, bad.n_cells = 12345, sp["mesh"].n_cells
        with pytest.raises(gpu.BielccError) as e:
            sv.submit_field(bad, sp["J"], sp["pts"], sp["k"])
        assert e.value.code == abi.ERR_NOT_FOUND
        # cancel a queued request
        sv.pause(True)
        t1 = _submit(sv, sp)
        t2 = _submit(sv, sp)
        sv.cancel(t2)
        sv.pause(False)
        assert sv.wait(t1)[0] == 0
        assert sv.wait(t2)[0] == abi.ERR_CANCELLED
        s = sv.stats()
        assert s["rejected"] == 1 and s["cancelled"] == 1
        assert 0 < s["peak_bytes_reserved"] <= s["budget"]
        # requests that do not fit the budget together run one after another
        # far points (no near pairs on this coarse mesh), ~2.7 MB reserved each (with the share of
        # the moments buffer): two exceed the budget
        pts = W.shell_points(300, 8.0, 10.0, np.random.default_rng(2))
        sv.pause(True)
        ta = sv.submit_field(sp["mesh"], sp["J"], pts, sp["k"])
        tb = sv.submit_field(sp["mesh"], sp["J"], pts, sp["k"])
        sv.pause(False)
        (sa, la, oa), (sb, lb, ob) = sv.wait(ta), sv.wait(tb)
        assert sa == sb == 0 and np.array_equal(oa["E"], ob["E"])
        assert sv.stats()["peak_bytes_reserved"] <= 4 << 20
    finally:
        sv.close()


def test_server_outputs_equal_the_batched_call(gctx):
    """Served complex64 results are the complex128 batched results rounded;
    served complex128 results are the batched results bit for bit."""
    torch = pytest.importorskip("torch")
    specs = _specs(gctx, 6)
    dev = torch.device("cuda:0")
    keep, jspecs = [], []
    for sp in specs:
        Jd = torch.from_numpy(np.ascontiguousarray(sp["J"])).to(dev)
        Pd = torch.from_numpy(np.ascontiguousarray(sp["pts"])).to(dev)
        S, P = sp["J"].shape[0], len(sp["pts"])
        Ed = torch.zeros((S, P, 3), dtype=torch.complex128, device=dev)
        Hd = torch.zeros_like(Ed)
        keep.append((Jd, Pd, Ed, Hd))
        jspecs.append(dict(mesh=sp["mesh"], n_rhs=S, n_pts=P, J=Jd.data_ptr(), pts=Pd.data_ptr(), E=Ed.data_ptr(),
                           H=Hd.data_ptr(), k=sp["k"], mult=sp["mult"]))
    gctx.field_EH_batch(gctx.make_jobs(jspecs), precision="mixed", stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    sv = gpu.Server(gctx, n_slots=2, precision="mixed")
    try:
        for sp, (_, _, Ed, Hd) in zip(specs, keep):
            E, H = Ed.cpu().numpy(), Hd.cpu().numpy()
            _, _, o64 = sv.wait(_submit(sv, sp, out_c64=False))
            _, _, o32 = sv.wait(_submit(sv, sp, out_c64=True))
            assert np.array_equal(o64["E"], E) and np.array_equal(o64["H"], H)
            assert np.array_equal(o32["E"], E.astype(np.complex64)) and np.array_equal(o32["H"], H.astype(np.complex64))
    finally:
        sv.close()


def test_server_concurrent_clients(gctx):
    """Four client threads submit and wait at the same time (host threads of
    one process, ctypes releasing the GIL); every result equals the same
    request served alone."""
    import threading

    specs = _specs(gctx, 7)
    sv = gpu.Server(gctx, n_slots=3, precision="mixed")
    try:
        alone = [sv.wait(_submit(sv, sp))[2] for sp in specs]
        errors = []

        def client(c):
            try:
                for rep in range(12):
                    i = (c + rep) % len(specs)
                    st, _, out = sv.wait(_submit(sv, specs[i]), timeout=120.0)
                    if st != 0 or not (np.array_equal(out["E"], alone[i]["E"]) and
                                       np.array_equal(out["H"], alone[i]["H"])):
                        errors.append((c, rep, st))
            except Exception as e:  # noqa: BLE001 - reported below
                errors.append((c, repr(e)))

        threads = [threading.Thread(target=client, args=(c,)) for c in range(4)]
        for t in threads:
            t.start()
        for t in threads:
            t.join(timeout=300)
        assert not errors, errors
        s = sv.stats()
        assert s["failed"] == 0 and s["completed"] == len(specs) + 48 and s["bytes_reserved"] == 0
    finally:
        sv.close()
