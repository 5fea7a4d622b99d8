"""Helpers shared by the GPU tests."""
import numpy as np
import torch

from argot_b200 import _lib as L
from argot_b200.pipeline import Problem, unit_box_grid
from oracle.oracle import unit_box_grid as orc_grid


def dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def march_segments(edge, fields, segs, precision, lunit=1.0, denstonh=1.0):
    lib = L.load()
    g = unit_box_grid(edge, lunit, denstonh)
    fd = [dev(f) for f in fields]
    packed = torch.empty(8 * edge ** 3, dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    L.check(lib.argot_b200_pack_fields(g, *(t.data_ptr() for t in fd), packed.data_ptr(), s), "pack")
    sd = dev(np.asarray(segs, np.float32))
    tau = torch.zeros(3 * len(segs), dtype=torch.float32, device="cuda")
    L.check(lib.argot_b200_march_segments(g, packed.data_ptr(), len(segs), sd.data_ptr(),
                                          tau.data_ptr(), int(precision), s), "march_segments")
    torch.cuda.synchronize()
    return tau.cpu().numpy().reshape(-1, 3)


def ray_segments(pb: Problem, emit, tgt):
    """Host restatement of the ray end points (calc_ray_segment.c:47-126 for
    sources inside the box): start = emitter position, end = the target cell
    centre xmin + ((float)i + 0.5)*delta in double, rounded to float."""
    pos4, _ = pb.emitters()
    start = pos4[emit, :3]
    d = np.float64(np.float32(1.0) / np.float32(pb.wl.edge))
    end = (0.0 + (tgt.astype(np.float32).astype(np.float64) + 0.5) * d).astype(np.float32)
    return np.concatenate([start, end], axis=1).astype(np.float32)


def run_problem(wl, precision, mode, max_group_rays=None):
    pb = Problem(wl, max_group_rays=max_group_rays)
    rays, tau = pb.alloc_group_buffers()
    rates = torch.zeros(6 * pb.ncell, dtype=torch.float32, device="cuda")
    taus, tables = [], []
    for gr in pb.groups:
        pb.emit(gr, rays)
        pb.march(gr, rays, tau, precision)
        pb.rates(gr, rays, tau, rates, mode)
        t = tau[:3 * gr.nray].view(3, gr.nray).t().cpu().numpy() if gr.nray else np.zeros((0, 3), np.float32)
        taus.append(t.copy())
        tables.append(pb.ray_table(rays, gr))
    torch.cuda.synchronize()
    pb.check_device_error()
    emit = np.concatenate([t[0] for t in tables])
    tgt = np.concatenate([t[1] for t in tables])
    return pb, emit, tgt, np.concatenate(taus), rates.view(6, -1).cpu().numpy()
