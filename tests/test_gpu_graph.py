"""The device-resident Fock build (qb_fock_device) captured into a CUDA graph
and replayed: after one warm-up call it allocates nothing and never waits for
the host, so one SCF iteration's two-electron step can be a graph.  Replays
with a new density (copied into the captured buffer) and a new cutMatrix
(uploaded with gpu_upload_cutoff_) must give the oracle's Fock matrix."""
import numpy as np
import pytest

from tests.helpers import case, random_density

pytestmark = pytest.mark.gpu


def test_fock_build_replays_from_a_cuda_graph(oracle_lib):
    import torch
    from quick_b200 import capi
    m, b = case("water4_631gs")
    n = b.nbasis
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    s = capi.Session(0)
    lib = capi.lib()
    try:
        s.upload_molecule(m, b, Y, cp)
        D0 = random_density(n, seed=7)
        cm0 = oracle_lib.cutmatrix(b, D0)
        s.get2e(np.zeros_like(D0), D0, cm0, 1e-10, 1e-20)    # uploads cutoffs, sizes the lists
        stream = torch.cuda.Stream()
        lib.qb_set_stream(capi.C.c_void_p(stream.cuda_stream))
        dD = torch.from_numpy(np.ascontiguousarray(D0)).cuda()
        dO = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        dOut = torch.empty_like(dO)
        ptr = lambda t: capi.C.c_void_p(t.data_ptr())  # noqa: E731
        with torch.cuda.stream(stream):
            assert lib.qb_fock_device(ptr(dD), ptr(dO), ptr(dOut)) == 0   # warm-up on this stream
        stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            rc = lib.qb_fock_device(ptr(dD), ptr(dO), ptr(dOut))
        assert rc == 0
        capi.check()
        for seed in (7, 11):
            D = random_density(n, seed=seed)
            cm = oracle_lib.cutmatrix(b, D)
            cmf = np.asfortranarray(cm)
            lib.gpu_upload_cutoff_(capi._ptr(cmf), capi._d(1e-10), capi._d(1e-20), None)
            torch.cuda.synchronize()
            dD.copy_(torch.from_numpy(np.ascontiguousarray(D)))
            g.replay()
            torch.cuda.synchronize()
            got = dOut.cpu().numpy()
            ref, _ = oracle_lib.fock(b, m.xyz_bohr, Y, cp, cm, D, 1e-10, 1e-20)
            assert np.abs(got - ref).max() < 1e-8
        del g
    finally:
        lib.qb_set_stream(capi.C.c_void_p(0))
        s.close()
