"""Helpers shared by the GPU tests: calls through the drop-in ``_C`` modules
(which call the C ABI) on numpy inputs, returning numpy outputs."""
import glob
import os

import numpy as np
import torch

from conftest import GOLDEN_DIR


def golden_cases(prefix):
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, prefix + "*.npz")))


def load_golden(name):
    with np.load(os.path.join(GOLDEN_DIR, name + ".npz")) as f:
        return {k: f[k] for k in f.files}


def cu(x, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    return t.to(dtype) if dtype is not None else t


def mf_forward(real, imag, tx, rx, voxel_3n, fs, As, precision, dtype=torch.float32, tuning=None):
    from geraf_b200.ops.RFMatchedFilter import _C

    A, S = real.shape
    N = voxel_3n.shape[1]
    out_r = torch.full((N,), float("nan"), dtype=dtype, device="cuda")
    out_i = torch.full((N,), float("nan"), dtype=dtype, device="cuda")
    _C.MatchedFilter_forward(cu(real, dtype), cu(imag, dtype), cu(tx, dtype), cu(rx, dtype), out_r,
                             out_i, cu(voxel_3n, dtype), A, S, float(fs), float(As), N,
                             precision=precision, tuning=tuning)
    torch.cuda.synchronize()
    return out_r.double().cpu().numpy(), out_i.double().cpu().numpy()


def mf_backward(gr, gi, tx, rx, voxel_3n, A, S, fs, As, precision, dtype=torch.float32, tuning=None):
    from geraf_b200.ops.RFMatchedFilter import _C

    N = voxel_3n.shape[1]
    g_r = torch.full((A, S), float("nan"), dtype=dtype, device="cuda")
    g_i = torch.full((A, S), float("nan"), dtype=dtype, device="cuda")
    dummy = torch.zeros((A, S), dtype=dtype, device="cuda")
    _C.MatchedFilter_backward_realimag(cu(gr, dtype), cu(gi, dtype), dummy, dummy, cu(tx, dtype),
                                       cu(rx, dtype), g_r, g_i, cu(voxel_3n, dtype), A, S, float(fs),
                                       float(As), N, precision=precision, tuning=tuning)
    torch.cuda.synchronize()
    return g_r.double().cpu().numpy(), g_i.double().cpu().numpy()


def tracer_forward(inp, S, precision, dtype=torch.float32, tuning=None):
    from geraf_b200.ops.RFSignalTracer import _C

    A, P = inp["sigmas"].shape
    t = {k: cu(inp[k], dtype) for k in ("normals", "sigmas", "points", "tx", "rx")}
    out_r = torch.full((A, S), float("nan"), dtype=dtype, device="cuda")
    out_i = torch.full((A, S), float("nan"), dtype=dtype, device="cuda")
    _C.SignalTracer_forward(t["normals"], t["sigmas"], t["points"], t["tx"], t["rx"],
                            cu(inp["inbounds"]).bool(), out_r, out_i, S, float(inp["fs"]),
                            float(inp["f0"]), float(inp["As"]), A, P, precision=precision,
                            tuning=tuning)
    torch.cuda.synchronize()
    return out_r.double().cpu().numpy(), out_i.double().cpu().numpy()


def tracer_backward(inp, gr, gi, precision, dtype=torch.float32, with_points=True, tuning=None):
    from geraf_b200.ops.RFSignalTracer import _C

    A, P = inp["sigmas"].shape
    S = gr.shape[1]
    t = {k: cu(inp[k], dtype) for k in ("normals", "sigmas", "points", "tx", "rx")}
    gn = torch.full((P, 3), float("nan"), dtype=dtype, device="cuda")
    gs = torch.full((A, P), float("nan"), dtype=dtype, device="cuda")
    gp = torch.full((P, 3), float("nan"), dtype=dtype, device="cuda") if with_points else None
    _C.SignalTracer_backward_normal_sigma(cu(gr, dtype), cu(gi, dtype), t["normals"], t["sigmas"],
                                          t["points"], t["tx"], t["rx"], cu(inp["inbounds"]).bool(),
                                          gn, gs, S, float(inp["fs"]), float(inp["f0"]),
                                          float(inp["As"]), A, P, grad_points=gp,
                                          precision=precision, tuning=tuning)
    torch.cuda.synchronize()
    out = [gn.double().cpu().numpy(), gs.double().cpu().numpy()]
    out.append(gp.double().cpu().numpy() if gp is not None else None)
    return out
