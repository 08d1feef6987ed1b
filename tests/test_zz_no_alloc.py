"""The zero-allocation sort entry point, nb_morton_sort_static.

It exists for callers that cannot let a library allocate device memory: a
renderer that steps the simulation every frame cannot take the device-wide
synchronisation cudaMalloc/cudaFree may cause, and applications that own all
device memory through their own pool pass buffers in instead.  The test hands
it device buffers it owns (allocated here through torch), checks that the
call changes no device allocation, and compares its codes, permutation and
box bit for bit with the context-based sort (nb_debug_morton) on two calls in
a row with different inputs.  This file is collected last on purpose.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NB_ERR_INVALID = 1
NB_ERR_CAPACITY = 3


def _device_buffers(torch, p):
    n = p.shape[0]
    dpos = torch.from_numpy(np.ascontiguousarray(p)).cuda()
    dcodes = torch.empty(n, dtype=torch.int64, device="cuda")
    dorder = torch.empty(n, dtype=torch.int32, device="cuda")
    dbox = torch.empty(4, dtype=torch.float64, device="cuda")
    return dpos, dcodes, dorder, dbox


def test_static_sort_matches_context_sort(nbp):
    torch = pytest.importorskip("torch")
    lib = nbp.load()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    cases = [nbp.universes.exponential_disc(200_000, 1),
             nbp.universes.colliding_discs(77_778, 2)]
    for m, p, v in cases:
        n = m.shape[0]
        dpos, dcodes, dorder, dbox = _device_buffers(torch, p)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = lib.nb_morton_sort_static(dpos.data_ptr(), n, dcodes.data_ptr(), dorder.data_ptr(),
                                       dbox.data_ptr(), stream.cuda_stream)
        assert rc == 0
        torch.cuda.synchronize()
        if free_before:
            # the first call on a device may load the library's device image;
            # from then on a call must leave device memory untouched
            rc = lib.nb_morton_sort_static(dpos.data_ptr(), n, dcodes.data_ptr(),
                                           dorder.data_ptr(), dbox.data_ptr(), stream.cuda_stream)
            assert rc == 0
            torch.cuda.synchronize()
            free_mid = torch.cuda.mem_get_info()[0]
            rc = lib.nb_morton_sort_static(dpos.data_ptr(), n, dcodes.data_ptr(),
                                           dorder.data_ptr(), dbox.data_ptr(), stream.cuda_stream)
            assert rc == 0
            torch.cuda.synchronize()
            assert torch.cuda.mem_get_info()[0] == free_mid
        codes = dcodes.cpu().numpy().view(np.uint64)
        order = dorder.cpu().numpy()
        box = dbox.cpu().numpy()
        with nbp.NbContext(nbp.SimConfig(), m, p, v) as ctx:
            codes_ref, order_ref, box_ref = ctx.debug_morton()
        assert np.array_equal(codes, codes_ref)
        assert np.array_equal(order, order_ref)
        assert np.array_equal(box, box_ref)


def test_static_sort_rejects_sizes_beyond_its_scratch(nbp):
    torch = pytest.importorskip("torch")
    lib = nbp.load()
    torch.cuda.set_device(0)
    dpos, dcodes, dorder, dbox = _device_buffers(torch, np.zeros((4, 2)))
    too_many = nbp.NB_STATIC_SORT_MAX_BODIES + 1
    assert lib.nb_morton_sort_static(dpos.data_ptr(), too_many, dcodes.data_ptr(),
                                     dorder.data_ptr(), dbox.data_ptr(), None) == NB_ERR_CAPACITY
    assert lib.nb_morton_sort_static(dpos.data_ptr(), 0, dcodes.data_ptr(), dorder.data_ptr(),
                                     dbox.data_ptr(), None) == NB_ERR_INVALID
