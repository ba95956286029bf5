"""Calculation-grid sizing and observed-map placement (host logic).

Restates the reference's MUDPACK sizing (nfgs_solver.py:73-177) and the
centred pad/crop placement (nfgs_solver.py:1593-1609) for the host side of
the B200 solver.  These are integer rules; the sizes they produce fix every
device buffer shape.
"""

from __future__ import annotations

import math

__all__ = ["mudpack_axis_size", "fortran_grid", "calculation_grid", "pad_or_crop_center"]


def mudpack_axis_size(n_obs: int) -> int:
    """Padded MUDPACK-friendly size 2*2^k+1 or 3*2^k+1 (nfgs_solver.py:73-84)."""
    n_obs = int(n_obs)
    if n_obs < 2:
        return max(1, n_obs)
    r = float(n_obs)
    e2 = math.ceil(math.log((r - 1.0) / 2.0) / math.log(2.0)) + 1
    e3 = math.ceil(math.log((r - 1.0) / 3.0) / math.log(2.0)) + 1
    return min(int(2 * (2 ** (e2 - 1)) + 1), int(3 * (2 ** (e3 - 1)) + 1))


def fortran_grid(nxo: int, nyo: int, nzo: int, symmetric_xy: bool = False) -> dict:
    """Calc sizes and pads of nfpt_fortran_grid (nfgs_solver.py:105-177)."""
    nx, ny, nz = mudpack_axis_size(nxo), mudpack_axis_size(nyo), mudpack_axis_size(nzo)
    if symmetric_xy:
        for name, n, o in (("x", nx, nxo), ("y", ny, nyo)):
            if n < o:
                raise ValueError(f"calculation size {n} is smaller than observed size {o}")
        if (nx - nxo) % 2 == 1:
            nx += 1
        if (ny - nyo) % 2 == 1:
            ny += 1
    return {"nx": nx, "ny": ny, "nz": nz, "bfx": (nx - nxo) // 2, "bfy": (ny - nyo) // 2, "bfz": nz - nzo}


def calculation_grid(nx: int, ny: int, nz: int, *, pad_calculation_domain=True,
                     calculation_domain_mode: str = "mudpack", padded_buffer_zone: bool = True) -> dict:
    """Calculation grid chosen by the constructor (nfgs_solver.py:771-819)."""
    if pad_calculation_domain is None:
        pad_calculation_domain = padded_buffer_zone
    mode = str(calculation_domain_mode).lower().replace("-", "_")
    if mode not in ("mudpack", "mudpack_legacy", "bottom_padding"):
        raise ValueError("calculation_domain_mode must be 'mudpack', 'mudpack_legacy', or "
                         f"'bottom_padding'; got {calculation_domain_mode!r}")
    if bool(pad_calculation_domain):
        if mode in ("mudpack", "mudpack_legacy"):
            g = fortran_grid(nx, ny, nz, symmetric_xy=(mode == "mudpack"))
            return {"nx": g["nx"], "ny": g["ny"], "nz": g["nz"], "pad_xy": (g["bfx"], g["bfy"])}
        bp = (nx + ny) // 6
        cnx, cny = nx + 2 * bp, ny + 2 * bp
        cnz = min(cnx, cny)
        if cnz < nz:
            raise ValueError("bottom_padding calculation height cannot contain the input z domain: "
                             f"input_Nz={nz}, calculated Nz={cnz}")
        return {"nx": cnx, "ny": cny, "nz": cnz, "pad_xy": (bp, bp)}
    return {"nx": nx, "ny": ny, "nz": nz, "pad_xy": (0, 0)}


def pad_or_crop_center(ny: int, nx: int, ty: int, tx: int) -> dict:
    """Source/destination windows of the centred pad/crop (nfgs_solver.py:1593-1609)."""
    sy0, sx0 = max(0, (ny - ty) // 2), max(0, (nx - tx) // 2)
    cny, cnx = min(ny, ty), min(nx, tx)
    dy0, dx0 = max(0, (ty - ny) // 2), max(0, (tx - nx) // 2)
    return {"sy0": sy0, "sx0": sx0, "dy0": dy0, "dx0": dx0, "cny": cny, "cnx": cnx}
