"""The oct-tree built on the device (argot_b200_dev_tree_build) equals the
host-built tree uploaded to the device (argot_b200_tree_build +
argot_b200_dev_tree_upload, pinned to the reference's construct_tree by the
walk tests) bit for bit: node count, every node field, the sorted source
list, the emitters' positions, FP64 spectra and bounding box; and the ray
counts of a tree walk with either tree agree."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _source_sets():
    from argot_b200 import workload as W
    from argot_b200.workload import photon_rates
    from argot_b200.pipeline import photon_counts
    rng = np.random.default_rng(17)
    out = []
    big = W.largest(edge=64, nsrc=4096, seed=5)  # 4096 clustered sources (only the sources are used)
    out.append(("clustered4096", big))
    out.append(("uniform16", W.plain(edge=32, nsrc=16, seed=3)))
    one = W.plain(edge=16, nsrc=1, seed=4)
    out.append(("one", one))
    dup = W.plain(edge=32, nsrc=40, seed=6)
    # coincident sources (equal keys at every level: depth-21 leaves with
    # several sources) and sources on the box faces
    dup.src_pos[10:20] = dup.src_pos[3]
    dup.src_pos[20:23] = np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [0.0, 0.999999, 0.5]], np.float32)
    out.append(("coincident40", dup))
    specs = []
    for name, wl in out:
        spec = photon_rates(photon_counts, wl.src_type, wl.src_param, wl.src_rate)
        specs.append((name, wl, np.ascontiguousarray(spec, np.float64)))
    return specs


@pytest.mark.parametrize("case", range(4))
def test_device_tree_equals_host_tree(cuda_ok, case):
    from argot_b200 import _lib as L
    from argot_b200.pipeline import unit_box_grid
    lib = L.load()
    name, wl, spec = _source_sets()[case]
    grid = unit_box_grid(wl.edge, wl.lunit, wl.denstonh)
    pos = np.ascontiguousarray(wl.src_pos, np.float32)
    n = len(pos)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    # host build + upload
    ht, hd = C.c_void_p(), C.c_void_p()
    L.check(lib.argot_b200_tree_build(C.byref(grid), n, pos.ctypes.data, spec.ctypes.data, float(wl.theta),
                                      C.byref(ht)), "tree_build")
    L.check(lib.argot_b200_dev_tree_upload(ht, C.byref(hd), st), "upload")
    # device build
    pos_d = torch.from_numpy(pos).cuda()
    spec_d = torch.from_numpy(spec).cuda()
    dd = C.c_void_p()
    L.check(lib.argot_b200_dev_tree_build(C.byref(grid), n, pos_d.data_ptr(), spec_d.data_ptr(),
                                          C.c_float(wl.theta), C.byref(dd), st), "dev_tree_build")

    def info(t):
        nn, ne = C.c_int(), C.c_int()
        b = np.zeros(6, np.float32)
        L.check(lib.argot_b200_dev_tree_info(t, C.byref(nn), C.byref(ne), b.ctypes.data), "info")
        return nn.value, ne.value, b

    def copy(t, nn, ne):
        p4 = np.zeros((ne, 4), np.float32)
        s64 = np.zeros((ne, 256))
        nodes = np.zeros((nn, 8), np.int32)
        sl = np.zeros(n, np.int32)
        L.check(lib.argot_b200_dev_tree_copy(t, p4.ctypes.data, s64.ctypes.data, nodes.ctypes.data,
                                             sl.ctypes.data, st), "copy")
        return p4, s64, nodes, sl

    nn, ne, bh = info(hd)
    nn2, ne2, bd = info(dd)
    assert (nn2, ne2) == (nn, ne) == (lib.argot_b200_tree_num_nodes(ht), lib.argot_b200_tree_num_emitters(ht))
    assert np.array_equal(bh, bd)
    h = copy(hd, nn, ne)
    d = copy(dd, nn, ne)
    for what, a, b in zip(("positions", "spectra", "nodes", "source list"), h, d):
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), (name, what)
    # the walk sees the same tree: ray counts per block
    nb = C.c_uint64()
    L.check(lib.argot_b200_num_blocks(C.byref(grid), C.byref(nb)), "num_blocks")
    counts = []
    for t in (hd, dd):
        c = torch.zeros(nb.value, dtype=torch.int64, device="cuda")
        L.check(lib.argot_b200_count_rays(C.byref(grid), t, 0, nb.value, c.data_ptr(), None, st), "count")
        torch.cuda.synchronize()
        counts.append(c.cpu().numpy())
    assert np.array_equal(counts[0], counts[1]) and counts[0].sum() > 0
    lib.argot_b200_dev_tree_free(hd)
    lib.argot_b200_dev_tree_free(dd)
    lib.argot_b200_tree_free(ht)
