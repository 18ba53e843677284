"""Host strip tiling of the TMA-tiled step (``cvfes_mesh_tiles``)."""
import numpy as np
import pytest

from cvfes_b200._lib import call, ptr
from cvfes_b200.cases import CASES, TubeCase
from cvfes_b200.mesh import special_assignment, tube_mesh
from cvfes_b200.plan import incidence


def tiles(elements, n_nodes, n_clamped, P, H, W, EH, WE):
    node_ptr, slot_rec, _ = incidence(elements, n_nodes)
    E = len(elements)
    nt = (n_nodes + P - 1) // P
    tw = np.empty((nt, W + WE), np.int32)
    tr = np.empty((3 * E, 4), np.int32)
    nl = np.empty(n_nodes, np.int32)
    st = np.zeros(4, np.int64)
    call("cvfes_mesh_tiles", n_nodes, E, ptr(node_ptr), ptr(slot_rec), n_clamped, P, H, W, EH,
         WE, ptr(tw), ptr(tr), ptr(nl), ptr(st))
    return node_ptr, slot_rec, tw, tr, nl, st


def resolve(loc, starts, h):
    """Id of a shared-memory row (or of a global reference)."""
    if loc < 0:
        return -1 - loc
    k, i = divmod(loc, h)
    assert starts[k] >= 0
    return starts[k] + i


@pytest.mark.parametrize("shape", [(16, 18, 3, 36, 2), (16, 18, 1, 36, 1), (8, 10, 4, 20, 3)])
def test_every_slot_row_resolves_to_its_id(lib, shape):
    P, H, W, EH, WE = shape
    case = TubeCase("tiles", 24, 12, 1.0)
    nodes, elems, inl, outl = tube_mesh(case.geometry())
    _, lel, _, nb = special_assignment(elems, len(nodes), np.concatenate([inl, outl]))
    N = len(nodes)
    node_ptr, slot_rec, tw, tr, nl, st = tiles(lel, N, nb, *shape)
    assert st[0] == len(tw)
    outl_n = outl_e = 0
    for a in range(nb, N):
        t = a // P
        ns, es = tw[t, :W], tw[t, W:]
        assert resolve(nl[a], ns, H) == a
        for k in range(node_ptr[a], node_ptr[a + 1]):
            e, b1, b2, fl = slot_rec[k]
            assert resolve(tr[k, 0], es, EH) == e
            assert resolve(tr[k, 1], ns, H) == b1 and resolve(tr[k, 2], ns, H) == b2
            assert tr[k, 3] == fl
            assert tr[k, 0] < WE * EH and max(tr[k, 1], tr[k, 2]) < W * H
            outl_e += int(tr[k, 0] < 0)
            outl_n += int(tr[k, 1] < 0) + int(tr[k, 2] < 0)
    assert st[1] == outl_n and st[2] == outl_e


def test_ring_numbered_tube_needs_few_windows(lib):
    """The 256x1024 tube: strips of 16 nodes have their neighbours in at most four windows
    of 18 ids, and with three windows almost nothing is left to global memory."""
    case = CASES["tube256x1024"]
    nodes, elems, inl, outl = tube_mesh(case.geometry())
    _, lel, _, nb = special_assignment(elems, len(nodes), np.concatenate([inl, outl]))
    _, slot_rec, tw, tr, nl, st = tiles(lel, len(nodes), nb, 16, 18, 3, 36, 2)
    refs = 2 * len(slot_rec)
    assert st[3] <= 4
    assert st[1] / refs < 1e-3 and st[2] / (refs / 2) < 2e-3


def test_bad_arguments_are_rejected(lib):
    from cvfes_b200._lib import CvfesError
    with pytest.raises(CvfesError):
        tiles(np.array([[0, 1, 2]]), 3, 0, 4, 2, 1, 4, 1)  # H < P


def test_numbering_bandwidth_leaves_out_the_clamped_prefix():
    """The solver's numbering puts both end rings first; the bandwidth that sets the L2
    prefetch distance is that of the unclamped nodes (one ring + 1 on the tube)."""
    from cvfes_b200.plan import numbering_bandwidth
    nc, na = 64, 128
    from cvfes_b200.mesh import TubeGeometry
    nodes, elems, inl, outl = tube_mesh(TubeGeometry(nc, na, 3.0))
    boundary = np.concatenate([inl, outl])
    assert numbering_bandwidth(elems, 0) == nc + 1
    _, lcl_elems, _, n_clamped = special_assignment(elems, nodes.shape[0], boundary)
    assert n_clamped == 2 * nc
    assert numbering_bandwidth(lcl_elems, n_clamped) == nc + 1
    assert numbering_bandwidth(lcl_elems, 0) > 50 * nc  # the last ring sits in the prefix
    assert numbering_bandwidth(np.array([[0, 1, 2]]), 3) == 0


def test_fan_item_shape_of_the_batch_kernel():
    """Nodes per warp of a batched fan item, the key the batch groups its meshes by."""
    from cvfes_b200.batched import fan_item_nodes
    assert [fan_item_nodes(S, 4) for S in (16, 32, 64, 128, 256, 200, 8)] == \
        [8, 4, 2, 1, 1, 1, 16]
    assert [fan_item_nodes(S, 1) for S in (16, 32, 64)] == [2, 1, 1]
