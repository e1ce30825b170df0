"""blaze_contact_list_static: the broad phase for callers that may not
allocate device memory.

A solver that calls this library between its own kernels (coupled CFD-DEM,
FEM) often cannot call cudaMalloc / cudaFree, which synchronise the device,
or owns all device memory through its own pool.  This entry point keeps its
working memory in a fixed array inside the library.  The test drives it
through the C ABI with caller-owned torch buffers and checks that it returns
exactly the contact list, cell order and status of the handle API's own
re-sort (blaze_get_nlist after one step), on two calls in a row: the second
call runs on a different state and must not see anything the first left in
the shared array.
"""
import ctypes as C

import numpy as np
import pytest

from blaze import device, synth
from blaze import types as T

pytestmark = pytest.mark.gpu

SKIN = 0.12   # cm; the lattice gap is ~0.1 cm, so every sphere has neighbours
CAP = 32


def static_entry():
    lib = device.load()
    f = lib.blaze_contact_list_static
    f.argtypes = [C.c_void_p, C.c_int, C.POINTER(T.SimulationInfo), C.c_float, C.c_int,
                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def handle_api_list(P, st):
    """Contact list of the step's own re-sort of state `st`."""
    sim = device.Simulation(P, skin=SKIN, max_nbr=CAP)
    sim.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
    sim.step(1)
    assert sim.sync() == 0
    nn, lst = sim.nlist()
    pid = sim.state()["pid"]
    sim.close()
    return nn, lst, pid


def static_list(f, P, st):
    import torch
    n = P.num_particles
    radius = np.array([P.pobj[t].radius for t in range(P.n_p)], np.float32)
    pos4 = np.concatenate([st["pos"].astype(np.float32), radius[st["type"]][:, None]], 1)
    d_pos4 = torch.from_numpy(np.ascontiguousarray(pos4)).cuda()
    # outputs start as garbage: the call must write every entry it reports
    perm = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    nn = torch.full((n,), 0x5EED, dtype=torch.int32, device="cuda")
    lst = torch.full((CAP, n), -1, dtype=torch.int32, device="cuda")
    status = torch.full((1,), 0x7777, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    rc = f(d_pos4.data_ptr(), n, C.byref(P.sim_info), SKIN, CAP, perm.data_ptr(), nn.data_ptr(),
           lst.data_ptr(), status.data_ptr(), stream.cuda_stream)
    assert rc == 0, rc
    stream.synchronize()
    nn_h = nn.cpu().numpy().view(np.uint32)
    slots = lst.cpu().numpy().view(np.uint32).T  # (n, CAP)
    live = np.arange(CAP)[None, :] < nn_h[:, None]
    return perm.cpu().numpy(), nn_h, np.where(live, slots, 0), int(status.item())


def test_static_scratch_matches_handle_api(tmp_path):
    # 5,120 spheres; cells of 2 r + skin, so that every pair within the skin
    # is searched and the handle API keeps the project's grid
    P, st0 = synth.box_project(str(tmp_path), n_side=(16, 16, 20), cell=0.32)
    f = static_entry()
    # a second, different state: the packing after 150 steps of settling,
    # stored in that run's (cell-sorted) order
    sim = device.Simulation(P)
    sim.set_state(st0["pos"], st0["vel"], st0["avel"], st0["type"], st0["pid"])
    sim.step(150)
    st1 = sim.state()
    assert st1["status"] == 0
    sim.close()
    for st in (st0, st1):
        nn_ref, lst_ref, pid_ref = handle_api_list(P, st)
        assert nn_ref.sum() > 0
        perm, nn, lst, status = static_list(f, P, st)
        assert status == 0, device.decode_status(status)
        np.testing.assert_array_equal(st["pid"][perm], pid_ref)
        np.testing.assert_array_equal(nn, nn_ref)
        np.testing.assert_array_equal(lst, lst_ref)


def test_static_scratch_rejects_sizes_beyond_its_limit(tmp_path):
    P, _ = synth.box_project(str(tmp_path), n_side=(4, 4, 4))
    f = static_entry()
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    assert f(dummy, 65537, C.byref(P.sim_info), SKIN, CAP, dummy, dummy, dummy, None, None) == -3
    si = T.SimulationInfo.from_buffer_copy(bytes(P.sim_info))
    si.num_NNCells = T.int3(100, 100, 100)   # 1,000,000 hash cells > 262,144
    assert f(dummy, 64, C.byref(si), SKIN, CAP, dummy, dummy, dummy, None, None) == -3


def test_static_cells_too_small_for_the_skin(tmp_path):
    """The box's own 0.2 cm cells with a 0.12 cm skin (2 r + skin = 0.32):
    pairs more than one cell edge apart are not searched, and the call says
    so with status 128."""
    P, st0 = synth.box_project(str(tmp_path), n_side=(16, 16, 20))
    f = static_entry()
    perm, nn, lst, status = static_list(f, P, st0)
    assert status & 128, device.decode_status(status)
