"""Per-batch registration wrappers, device-resident.

``wbi_registration_3d`` and ``wbi_registration_2d`` keep the signatures,
config keys, outputs and layouts of the reference's
``utils/registration.py:41-352``: the template (given, or picked from the
batch by ``pick_initial_reference``, ``utils/reference.py:19-99``), the
optional dual-channel mix (``transform``, ``utils/registration.py:28-38``),
the outlier masks of the template and of every frame (``getMask`` +
``bwareafilt3_wei``), the smoothness-penalty normalisation, then per frame
``getMotion`` and ``correctMotion`` of the membrane channel, the calcium
channel and the mixed frame, with the mean squared error before and after.
Every step runs on the GPU: the registration and the masks in the sm_100a
library, the template picking's frame-by-frame correlation as the
library's demeaned Gram kernel (``wr_frame_gram``, float64 sums).  Inputs
may be NumPy arrays (returned as NumPy, like the
reference) or CUDA tensors (returned as CUDA tensors).
"""

from __future__ import annotations

import os

import numpy as np
import torch

from . import _lib

from .mask import bwareafilt3_wei, getMask
from .registrar import LKParams, LKRegistrar, penalty_factor, warp

# the package-level option["zRatio"] default (utils/__init__.py:83), used when
# the config carries no MetaData.zRatio, and always by the 2-D wrapper
DEFAULT_ZRATIO = 27.693

_REG_DTYPES = (torch.uint8, torch.uint16, torch.float32)


def _load_config(config_file):
    if isinstance(config_file, dict):
        return config_file
    import tomllib

    with open(os.fspath(config_file), "rb") as fh:
        return tomllib.load(fh)


def transform(image, k=1, method="raw"):
    """utils/registration.py:28-38 on tensors."""
    if method == "raw":
        return k * image
    if method == "sqrt":
        return k * torch.sqrt(image)
    if method == "log2":
        return k * torch.log2(1 + image)
    if method == "log10":
        return k * torch.log10(1 + image)
    raise ValueError(f"Unknown method to process the image:{method}")


def pick_initial_reference(frames: torch.Tensor, max_corr_frames: int = 20, spatial_ds: int = 4):
    """utils/reference.py:19-99 on the device: the frames' correlation matrix
    over the central three z planes (x and y subsampled by ``spatial_ds``)
    from the library's demeaned Gram kernel (the reference's float32 GEMM,
    summed here in float64), the frame whose ``max_corr_frames`` best correlations
    have the largest mean, and the full-resolution mean of that frame's best
    correlated frames.  Returns (reference, indices)."""
    if frames.dim() == 4:
        T, Z = frames.shape[:2]
        used = frames[:, Z // 2 - 1:Z // 2 + 2] if Z >= 3 else frames
    elif frames.dim() == 3:
        T = frames.shape[0]
        used = frames[:, None]
    else:
        raise ValueError("frames must be [T,Y,X] or [T,Z,Y,X]")
    small = used[:, :, ::spatial_ds, ::spatial_ds].to(torch.float32).contiguous()
    if not small.is_cuda:
        raise ValueError("pick_initial_reference runs on a CUDA device: frames must be a CUDA tensor")
    flat = small.reshape(T, -1)
    # the demeaned frames' Gram matrix (the reference's float32 GEMM), summed in float64 by wr_frame_gram
    lib = _lib.load()
    means = torch.empty(T, dtype=torch.float64, device=flat.device)
    cc = torch.empty((T, T), dtype=torch.float64, device=flat.device)
    _lib.check("wr_frame_gram", lib.wr_frame_gram(flat.data_ptr(), T, flat.shape[1], means.data_ptr(), cc.data_ptr(),
                                                  torch.cuda.current_stream(flat.device).cuda_stream))
    diag = torch.sqrt(torch.diagonal(cc)) + 1e-12
    cc = cc / (diag[:, None] * diag[None, :])
    ncorr = min(max_corr_frames, T - 1)
    if ncorr < 1:
        idx = torch.arange(T, device=frames.device)
        return _mean_of(frames, idx), idx
    ccsort = torch.sort(cc, dim=1, descending=True).values
    best = ccsort[:, 1:ncorr + 1].mean(dim=1)
    imax = int(torch.argmax(best).item())
    top = torch.argsort(-cc[imax], stable=True)[:ncorr]
    return _mean_of(frames, top), top


def _mean_of(frames, idx):
    """Mean of frames[idx] over the first axis with NumPy's dtype rules, the
    frames added in index order as NumPy's axis-0 mean adds them: float32
    (and float16, through a float32 sum) frames keep their type, every other
    type is averaged in float64."""
    if frames.dtype in (torch.float32, torch.float16):
        acc_t, out_t = torch.float32, frames.dtype
    else:
        acc_t, out_t = torch.float64, torch.float64
    acc = None
    for i in idx.tolist():
        f = frames[int(i)].to(acc_t)
        acc = f if acc is None else acc + f
    return (acc / len(idx)).to(out_t)


def compute_reference_from_block(mem_block, config, ca_block=None):
    """utils/reference.py:102-124: the reference of a block of frames.

    The mean of the frames best correlated with the most representative one
    (pick_initial_reference with min(T // 2, 50) correlations), plus, for
    dual-channel data with k != 0, the transformed float64 mean of the second
    channel over the same frames.  mem_block / ca_block: [T, Z, Y, X] or
    [T, Y, X] NumPy arrays (moved to the current CUDA device, as the
    reference moves them to its GPU) or tensors (used where they are).
    Returns (reference, indices) as NumPy arrays, as the reference does."""
    channels = config["channels"]
    k, function, dual = channels["k"], channels["function"], channels["dual_channel"]
    n_corr = min(len(mem_block) // 2, 50)
    device = mem_block.device if isinstance(mem_block, torch.Tensor) else _device(None)
    mem = _as_tensor(mem_block, device)
    mem_ref, indsort = pick_initial_reference(mem, max_corr_frames=n_corr)
    result = mem_ref
    if dual and k != 0:
        if ca_block is None:
            raise ValueError("ca_block is required for dual-channel data with k != 0")
        ca_ref = _mean_of(_as_tensor(ca_block, device), indsort)
        result = mem_ref + transform(ca_ref, k, function)
    return result.cpu().numpy(), indsort.cpu().numpy()


def _mse(a, b) -> float:
    """np.mean((a - b) ** 2) with NumPy's dtype rules: two arrays of one
    unsigned integer type subtract and square with wrap-around (as the
    reference's uint16 frames and template do); otherwise the values are
    squared in float64 here (NumPy: in the promoted float type)."""
    if a.dtype == b.dtype and a.dtype in (torch.uint8, torch.uint16):
        mod = 1 << (8 * a.element_size())
        d = (a.to(torch.int64) - b.to(torch.int64)) % mod
        return float(((d * d) % mod).to(torch.float64).mean().item())
    return float(((a.to(torch.float64) - b.to(torch.float64)) ** 2).mean().item())


def _as_tensor(a, device):
    if a is None:
        return None
    if isinstance(a, torch.Tensor):
        return a.to(device)
    return torch.from_numpy(np.ascontiguousarray(a)).to(device)


def _reg_dtype(t):
    return t if t.dtype in _REG_DTYPES else t.to(torch.float32)


def _template(mem, ca, reference_image, config, device):
    """The template (given, or picked from the frames) plus, for dual-channel
    runs with a picked template, the transformed calcium template's mean and
    std (utils/registration.py:215-246)."""
    refer = config["reference"]
    channels = config["channels"]
    if refer["pick_reference_auto"]:
        membrane_ref, indsort = pick_initial_reference(mem, max_corr_frames=refer["chunk_size"])
    else:
        if reference_image is None:
            raise ValueError("reference_image is required when reference.pick_reference_auto is false")
        membrane_ref = _as_tensor(reference_image, device)
        indsort = None
    if channels["dual_channel"] and ca is None:
        raise ValueError("[ERROR] Calcium image stack shouldn't be empty")
    if channels["dual_channel"] and refer["pick_reference_auto"] and channels["k"] != 0:
        ca_ref = _mean_of(ca, indsort)
        ca_ref_t = transform(ca_ref, channels["k"], channels["function"])
        return membrane_ref.to(torch.float64) + ca_ref_t, ca_ref_t.mean(), ca_ref_t.std(unbiased=False)
    return membrane_ref, None, None


def _register_frames(mem, ca, dat_ref, ref_mean, ref_std, config, zratio, motion_init, verbose, frame, device):
    """Masks, penalty factor, then per frame getMotion + correctMotion and the
    errors (utils/registration.py:252-346); frames (T, Z, Y, X)."""
    channels = config["channels"]
    refer = config["reference"]
    dual = channels["dual_channel"]
    mcfg = config["mask"]
    mask_range, thres = mcfg["maskRange"], mcfg["thresFactor"]
    dat_ref = dat_ref.contiguous()
    mask_ref = bwareafilt3_wei(getMask(_reg_dtype(dat_ref), thres), mask_range)
    pyr = config["pyramid"]
    # one dtype for the registration: the frames' own when the template shares it, else float32
    same_int = dat_ref.dtype == mem.dtype and mem.dtype in (torch.uint8, torch.uint16) and not dual
    ref_reg = dat_ref if same_int else dat_ref.to(torch.float32)
    factor = float(penalty_factor(ref_reg, mask_ref).item())
    params = LKParams(layer=int(pyr["layer"]), iter=int(pyr["iter"]), r=int(pyr["r"]), zRatio=float(zratio),
                      movRange=5.0, smoothPenalty=factor * float(pyr["smoothPenalty"]), tol=float(pyr["tolerance"]))
    shape = tuple(mem.shape[1:])
    reg = LKRegistrar(shape, params, device)
    init = _as_tensor(motion_init, device)
    if init is not None:
        init = init.to(torch.float32).contiguous()

    mem_out, ca_out, errors, motions = [], [], [], []
    for i in range(mem.shape[0]):
        dat_mem = mem[i].contiguous()
        if dual:
            dat_ca = ca[i].contiguous()
            ca_t = transform(dat_ca.to(torch.float64), channels["k"], channels["function"])
            if refer["pick_reference_auto"] and ref_mean is not None:
                # prep.normalize_std (utils/preprocess.py:288-293)
                ca_t = (ca_t - ca_t.mean()) / ca_t.std(unbiased=False) * ref_std + ref_mean
            dat_mov = dat_mem.to(torch.float64) + ca_t
        else:
            dat_mov = dat_mem
        mov_reg = dat_mov if same_int else dat_mov.to(torch.float32).contiguous()
        mask_mov = bwareafilt3_wei(getMask(mov_reg, thres), mask_range)
        corrected_mov = torch.empty(shape, dtype=torch.float32, device=device)
        motion = reg.register(mov_reg, ref_reg, mask_mov, mask_ref, motion_init=init, warped_out=corrected_mov)
        corrected_mem = corrected_mov if not dual else warp(_reg_dtype(dat_mem).contiguous(), motion)
        if dual:
            ca_out.append(warp(_reg_dtype(dat_ca).contiguous(), motion))
        initial = _mse(dat_mov, dat_ref)
        eventual = _mse(corrected_mov, dat_ref)
        if verbose:
            tag = i + 1 if frame is None else frame[i]
            print(f"        Frame: {tag}\tInitial Error is:{initial:.4f}\tEventual Error: {eventual:.4f}")
        errors.append({"initial_error": initial, "eventual_error": eventual})
        mem_out.append(corrected_mem.clone())
        motions.append(motion.clone())
    return (torch.stack(mem_out), torch.stack(ca_out) if ca_out else None, errors, torch.stack(motions), dat_ref)


def _device(device):
    return torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())


def wbi_registration_3d(moving_membrane_image, config_file, reference_image=None, motion_init=None, verbose=True,
                        frame=None, direction="forward", moving_Ca_image=None, device=None):
    """Register a batch of frames (T, Z, Y, X) (or one (Z, Y, X) frame).

    Returns ``(mem_out, ca_out, dat_ref, errors, motion_out)`` as the
    reference does: corrected membrane frames (T, Z, Y, X), corrected calcium
    frames (or an empty array), the template in (x, y, z) order, per-frame
    ``{"initial_error", "eventual_error"}`` and motions (T, Z, Y, X, 3)."""
    config = _load_config(config_file)
    to_numpy = not isinstance(moving_membrane_image, torch.Tensor)
    device = _device(device)
    mem = _as_tensor(moving_membrane_image, device)
    ca = _as_tensor(moving_Ca_image, device)
    if mem.dim() == 3:
        mem = mem[None]
        ca = ca[None] if ca is not None else None
    if mem.dim() != 4:
        raise ValueError("moving_membrane_image must be 3D or 4D array")
    dat_ref, ref_mean, ref_std = _template(mem, ca, reference_image, config, device)
    zratio = config.get("MetaData", {}).get("zRatio", DEFAULT_ZRATIO)
    mem_t, ca_t, errors, mot_t, dat_ref = _register_frames(mem, ca, dat_ref, ref_mean, ref_std, config, zratio,
                                                            motion_init, verbose, frame, device)
    if to_numpy:
        return (mem_t.cpu().numpy(), ca_t.cpu().numpy() if ca_t is not None else np.array([]),
                dat_ref.cpu().numpy().transpose(2, 1, 0), errors, mot_t.cpu().numpy())
    return mem_t, ca_t, dat_ref.permute(2, 1, 0), errors, mot_t


def wbi_registration_2d(moving_membrane_image, config_file, reference_image=None, motion_init=None, verbose=True,
                        frame=None, direction="forward", moving_Ca_image=None, device=None):
    """utils/registration.py:41-189: frames (T, Ly, Lx) registered as
    volumes of two identical planes.  As in the reference, the first image
    axis plays the role of x and the package default zRatio applies.

    Returns ``(mem_out, ca_out, dat_ref, errors, motion_out)``: corrected
    frames (T, Ly, Lx), calcium frames or an empty array, the stacked template
    (Ly, Lx, 2), errors, and motions (T, Ly, Lx, 3)."""
    config = _load_config(config_file)
    to_numpy = not isinstance(moving_membrane_image, torch.Tensor)
    device = _device(device)
    mem = _as_tensor(moving_membrane_image, device)
    ca = _as_tensor(moving_Ca_image, device)
    if mem.dim() == 2:
        mem = mem[None]
        ca = ca[None] if ca is not None else None
    if mem.dim() != 3:
        raise ValueError("moving_membrane_image must be 2D or 3D array")
    ref_1plane, ref_mean, ref_std = _template(mem, ca, reference_image, config, device)
    # a reference (d0, d1, 2) array, (x, y, z) to it, is the (2, d1, d0) volume here
    as_vol = lambda img: torch.stack([img.transpose(-1, -2)] * 2, dim=-3).contiguous()
    init = None
    if motion_init is not None:
        m = _as_tensor(motion_init, device).to(torch.float32)     # (d0, d1, 3)
        init = torch.stack([m.transpose(0, 1)] * 2, dim=0).contiguous()
    mem_t, ca_t, errors, mot_t, _ = _register_frames(
        as_vol(mem), as_vol(ca) if ca is not None else None, as_vol(ref_1plane), ref_mean, ref_std, config,
        DEFAULT_ZRATIO, init, verbose, frame, device)
    mem2 = mem_t[:, 0].transpose(1, 2)
    ca2 = ca_t[:, 0].transpose(1, 2) if ca_t is not None else None
    mot2 = mot_t[:, 0].transpose(1, 2)
    dat_ref = torch.stack([ref_1plane] * 2, dim=2)
    if to_numpy:
        return (mem2.cpu().numpy(), ca2.cpu().numpy() if ca2 is not None else np.array([]), dat_ref.cpu().numpy(),
                errors, mot2.cpu().numpy())
    return mem2, ca2, dat_ref, errors, mot2
