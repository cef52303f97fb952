"""The allocation-free H*psi entry point (pspw_apply_ham_block_dev_noalloc).

It exists for callers that cannot let the library allocate device memory
while it is being called -- code recorded into a CUDA graph, programs whose
memory manager owns the whole device, services that must not run out of
memory in mid-request -- and takes its scratch from a fixed 16 MiB array in
the library instead.  These tests call it through the C ABI and compare it
with the allocating entry point, twice in a row (the shared array keeps the
first call's contents, which must not leak into the second), and check that
the second call leaves the device's free memory unchanged.

The file name sorts last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from helpers import relmax  # noqa: E402
from pspw import PREC_F32, PREC_F64, Cell, PspwError, basis_gamma, synth, workloads  # noqa: E402
from pspw._lib import check, lib, ptr  # noqa: E402


@pytest.fixture(scope="module")
def si8():
    w = workloads.workload("si8")
    cell = workloads.make_cell(w)
    return w, cell


def _noalloc(cell, d_in, d_out, ld, ngw, nb, prec):
    check(lib().pspw_apply_ham_block_dev_noalloc(cell.handle, prec, ptr(d_in), ptr(d_out), ld,
                                                 ngw, nb))


def _alloc(cell, d_in, d_out, ld, ngw, nb, prec):
    check(lib().pspw_apply_ham_block_dev(cell.handle, prec, ptr(d_in), ptr(d_out), ld, ngw, nb))


@pytest.mark.parametrize("prec,dtype,tol", [(PREC_F64, torch.complex128, 1e-12),
                                            (PREC_F32, torch.complex64, 2e-5)])
def test_noalloc_matches_allocating_entry_point_twice(si8, prec, dtype, tol):
    w, cell = si8
    psi = w["psi"]
    ngw, nb = psi.shape
    d_in = torch.from_numpy(np.ascontiguousarray(psi.T)).to(dtype).cuda()
    ref = torch.zeros_like(d_in)
    torch.cuda.synchronize()
    _alloc(cell, d_in, ref, ngw, ngw, nb, prec)
    check(lib().pspw_cell_synchronize(cell.handle))
    expect = ref.cpu().numpy()
    for call in range(2):
        out = torch.full_like(d_in, float("nan"))
        torch.cuda.synchronize()
        _noalloc(cell, d_in, out, ngw, ngw, nb, prec)
        check(lib().pspw_cell_synchronize(cell.handle))
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got)), f"call {call}"
        assert relmax(got, expect) < tol, f"call {call}"


@pytest.mark.parametrize("prec,dtype,tol", [(PREC_F64, torch.complex128, 1e-12),
                                            (PREC_F32, torch.complex64, 2e-5)])
def test_noalloc_generic_fft_grid_twice(prec, dtype, tol):
    # a 22 x 21 x 26 grid (radices 2, 3, 7, 11, 13) is outside the register
    # FFT: the general passes run with their stick and plane buffers placed
    # in the static array by the same plan
    lat, pos = synth.si_diamond(1)
    b = basis_gamma(lat, 8.0, (22, 21, 26), [8], [pos])
    pkg_a, wnl = synth.kb_form_factors(b, lat)
    b.update(pkg_a=pkg_a, wnl=wnl, lm_end=[4])
    cell = Cell.from_arrays(b)
    cell.set_veff(synth.local_potential(b["nr"], lat, pos))
    psi = synth.wavefunctions(b, lat, 7, 3)
    ngw, nb = psi.shape
    d_in = torch.from_numpy(np.ascontiguousarray(psi.T)).to(dtype).cuda()
    ref = torch.zeros_like(d_in)
    torch.cuda.synchronize()
    _alloc(cell, d_in, ref, ngw, ngw, nb, prec)
    check(lib().pspw_cell_synchronize(cell.handle))
    expect = ref.cpu().numpy()
    for call in range(2):
        out = torch.full_like(d_in, float("nan"))
        torch.cuda.synchronize()
        _noalloc(cell, d_in, out, ngw, ngw, nb, prec)
        check(lib().pspw_cell_synchronize(cell.handle))
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got)), f"call {call}"
        assert relmax(got, expect) < tol, f"call {call}"


@pytest.mark.parametrize("prec,dtype,tol", [(PREC_F64, torch.complex128, 1e-12),
                                            (PREC_F32, torch.complex64, 2e-5)])
def test_noalloc_call_captured_in_a_cuda_graph(si8, prec, dtype, tol):
    """The entry point recorded into a CUDA graph on the cell stream (relaxed
    capture mode) after one eager warm-up call; the graph replayed twice
    gives the eager result both times."""
    rt = C.CDLL("libcudart.so.12")  # the runtime the library is linked with
    w, cell = si8
    psi = w["psi"]
    ngw, nb = psi.shape
    d_in = torch.from_numpy(np.ascontiguousarray(psi.T)).to(dtype).cuda()
    ref = torch.zeros_like(d_in)
    out = torch.zeros_like(d_in)
    torch.cuda.synchronize()
    _alloc(cell, d_in, ref, ngw, ngw, nb, prec)
    _noalloc(cell, d_in, out, ngw, ngw, nb, prec)  # warm-up
    check(lib().pspw_cell_synchronize(cell.handle))
    expect = ref.cpu().numpy()
    st = C.c_void_p(cell.stream())
    graph, gexec = C.c_void_p(), C.c_void_p()
    assert rt.cudaStreamBeginCapture(st, 2) == 0  # cudaStreamCaptureModeRelaxed
    try:
        _noalloc(cell, d_in, out, ngw, ngw, nb, prec)
    finally:
        end = rt.cudaStreamEndCapture(st, C.byref(graph))
    assert end == 0
    assert rt.cudaGraphInstantiate(C.byref(gexec), graph, C.c_ulonglong(0)) == 0
    try:
        for rep in range(2):
            out.fill_(float("nan"))
            torch.cuda.synchronize()
            assert rt.cudaGraphLaunch(gexec, st) == 0
            assert rt.cudaStreamSynchronize(st) == 0
            got = out.cpu().numpy()
            assert np.all(np.isfinite(got)), f"replay {rep}"
            assert relmax(got, expect) < tol, f"replay {rep}"
    finally:
        rt.cudaGraphExecDestroy(gexec)
        rt.cudaGraphDestroy(graph)


def test_noalloc_second_call_leaves_free_memory_unchanged(si8):
    w, cell = si8
    psi = w["psi"][:, :5]
    ngw = psi.shape[0]
    d_in = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda()
    d_out = torch.zeros_like(d_in)
    torch.cuda.synchronize()
    _noalloc(cell, d_in, d_out, ngw, ngw, 5, PREC_F64)  # first call: address look-up
    check(lib().pspw_cell_synchronize(cell.handle))
    free0, _ = torch.cuda.mem_get_info()
    _noalloc(cell, d_in, d_out, ngw, ngw, 5, PREC_F64)
    check(lib().pspw_cell_synchronize(cell.handle))
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_blocks_beyond_the_static_scratch():
    # the Si216 cell (96^3 grid) needs ~2.3 MB of FFT scratch per band and
    # 864 projectors: a 512-band block's projection buffers alone exceed it
    w = workloads.si_cell(3, 96, with_veff=False)
    from pspw import Cell
    cell = Cell.from_arrays(w)
    ngw = w["ngw"]
    nb = 512
    d = torch.zeros((nb, ngw), dtype=torch.complex128, device="cuda")
    o = torch.zeros_like(d)
    veff = torch.zeros(int(np.prod(w["nr"])), dtype=torch.float64, device="cuda")
    check(lib().pspw_cell_set_veff_device(cell.handle, ptr(veff), veff.numel()))
    with pytest.raises(PspwError) as e:
        _noalloc(cell, d, o, ngw, ngw, nb, PREC_F64)
    assert e.value.code == 2 and "16 MiB" in str(e.value)
