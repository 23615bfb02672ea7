"""Post-processing of the solver's output files (the reference's post/ layer).

`profile_metrics` and `profile_objective` restate the mean-profile
quantities of post/plot_profiles.py (centreline velocity, half-width) for the
time-averaged radial statistics; the jet adjoint's profile objective uses the
same definitions (mcg_adjoint_jet_profile_run).

`write_uy_avg_vti` replaces post/binConversionVti.py:12-51, which needs the
`vtk` package to turn `mean_profiles/uy_avg.bin` (float32, NX*NY*NZ, x
fastest) into `profiles/uy_avg.vti`.  This one writes the same VTK XML
ImageData file as plain text: one Float32 point array named `uy_avg`, inline
binary (base64 of [UInt64 byte count][payload], the format of the solver's
own `vti_data/lbm_*.vti`).  ParaView and vtkXMLImageDataReader read it.  The
grid size comes from the case directory's `case_info.txt`, so no
`constants.cuh` is needed.

    python -m multicomponent_color_gradient_b200.post --case-dir JET_VTK/Re120_We8
"""
from __future__ import annotations

import argparse
import base64
import struct
from pathlib import Path
from typing import Dict, Optional, Union

import numpy as np

PathLike = Union[str, Path]


def read_case_info(case_dir: PathLike) -> Dict[str, str]:
    """Key/value lines of `<case_dir>/case_info.txt` (written by mcg_output_open)."""
    out: Dict[str, str] = {}
    for line in (Path(case_dir) / "case_info.txt").read_text().splitlines():
        parts = line.split(maxsplit=1)
        if len(parts) == 2:
            out[parts[0]] = parts[1]
    return out


def vti_text(nx: int, ny: int, nz: int, arrays: Dict[str, np.ndarray]) -> str:
    """VTK XML ImageData text with float32 point arrays, inline base64 with UInt64 headers."""
    ext = f"0 {nx - 1} 0 {ny - 1} 0 {nz - 1}"
    first = next(iter(arrays))
    parts = ['<?xml version="1.0"?>\n',
             '<VTKFile type="ImageData" version="1.0" byte_order="LittleEndian" header_type="UInt64">\n',
             f'  <ImageData WholeExtent="{ext}" Origin="0 0 0" Spacing="1 1 1">\n',
             f'    <Piece Extent="{ext}">\n',
             f'      <PointData Scalars="{first}">\n']
    for name, a in arrays.items():
        payload = np.ascontiguousarray(a, dtype="<f4").tobytes()
        text = base64.b64encode(struct.pack("<Q", len(payload)) + payload).decode("ascii")
        parts.append(f'        <DataArray type="Float32" Name="{name}" format="binary">\n{text}\n'
                     '        </DataArray>\n')
    parts.append("      </PointData>\n      <CellData>\n      </CellData>\n    </Piece>\n  </ImageData>\n"
                 "</VTKFile>\n")
    return "".join(parts)


def write_uy_avg_vti(case_dir: PathLike, output_dir: Optional[PathLike] = None) -> Path:
    """`<case_dir>/mean_profiles/uy_avg.bin` -> `<output_dir or case_dir/profiles>/uy_avg.vti`.

    Raises ValueError when the file does not hold NX*NY*NZ values, as
    post/binConversionVti.py:28-30 does."""
    case_dir = Path(case_dir)
    info = read_case_info(case_dir)
    nx, ny, nz = int(info["NX"]), int(info["NY"]), int(info["NZ"])
    input_path = case_dir / "mean_profiles" / "uy_avg.bin"
    data = np.fromfile(input_path, dtype="<f4")
    expected = nx * ny * nz
    if data.size != expected:
        raise ValueError(f"{input_path} has {data.size} values, expected {expected}")
    profiles_dir = Path(output_dir) if output_dir is not None else case_dir / "profiles"
    profiles_dir.mkdir(parents=True, exist_ok=True)
    output_path = profiles_dir / "uy_avg.vti"
    output_path.write_text(vti_text(nx, ny, nz, {"uy_avg": data}))
    print(f"uy_avg VTI written to {output_path}")
    return output_path


def radial_bin_radii(nx: int, nz: int, nr: int, x0: float, z0: float) -> np.ndarray:
    """Mean distance from the jet axis of the interior columns of each radial
    bin, 0 for the first (the numerical centreline), as
    post/plot_profiles.py:73-91 forms it."""
    rsum = np.zeros(nr)
    cnt = np.zeros(nr, np.int64)
    for x in range(1, nx - 1):
        for z in range(1, nz - 1):
            r = float(np.sqrt((float(x) - x0) ** 2 + (float(z) - z0) ** 2))
            rb = int(r)
            if rb < nr:
                rsum[rb] += r
                cnt[rb] += 1
    radius = np.arange(nr, dtype=np.float64)
    np.divide(rsum, cnt, out=radius, where=cnt > 0)
    radius[0] = 0.0
    return radius


def half_width(profile: np.ndarray, radius: np.ndarray, center_value: float) -> float:
    """First radius where profile/center_value falls to 1/2, interpolated
    linearly between bins; NaN when undefined (post/plot_profiles.py:53-70)."""
    if not np.isfinite(center_value) or center_value <= 0.0:
        return float("nan")
    ratio = profile / center_value
    below = np.where(np.isfinite(ratio) & (ratio <= 0.5))[0]
    below = below[below > 0]
    if below.size == 0:
        return float("nan")
    i = int(below[0])
    r1, r2, u1, u2 = radius[i - 1], radius[i], ratio[i - 1], ratio[i]
    if not np.isfinite(u1) or not np.isfinite(u2) or np.isclose(u1, u2):
        return float("nan")
    return float(r1 + (0.5 - u1) * (r2 - r1) / (u2 - u1))


def profile_metrics(sum_uy: np.ndarray, count: np.ndarray, nx: int, nz: int, x0: float, z0: float):
    """Centreline velocity uc[y] (the first annulus) and half-width r_half[y]
    of the time-averaged radial profiles sum_uy/count ((NY, NR_BINS) or flat)."""
    nr = nx // 2
    s = np.asarray(sum_uy, np.float64).reshape(-1, nr)
    c = np.asarray(count, np.float64).reshape(-1, nr)
    U = np.full(s.shape, np.nan)
    np.divide(s, c, out=U, where=c > 0)
    radius = radial_bin_radii(nx, nz, nr, x0, z0)
    uc = U[:, 0].copy()
    rh = np.array([half_width(U[y], radius, uc[y]) for y in range(U.shape[0])])
    return uc, rh


def profile_objective(uc, rh, uc_target, rh_target, y_lo: int, y_hi: int, u_jet: float, diameter: float) -> float:
    """J = 1/2 sum_{y_lo <= y <= y_hi} ((uc - uc*)/U)^2 + ((r_half - r_half*)/D)^2,
    each term where both of its values are defined."""
    J = 0.0
    for y in range(y_lo, y_hi + 1):
        if np.isfinite(uc[y]) and np.isfinite(uc_target[y]):
            J += 0.5 * ((float(uc[y]) - float(uc_target[y])) / u_jet) ** 2
        if np.isfinite(rh[y]) and np.isfinite(rh_target[y]):
            J += 0.5 * ((float(rh[y]) - float(rh_target[y])) / diameter) ** 2
    return J


def main() -> None:
    ap = argparse.ArgumentParser(description="Convert mean_profiles/uy_avg.bin to profiles/uy_avg.vti.")
    ap.add_argument("--case-dir", required=True, help="case directory, e.g. JET_VTK/Re120_We8")
    ap.add_argument("--output-dir", default=None, help="defaults to <case-dir>/profiles")
    args = ap.parse_args()
    write_uy_avg_vti(args.case_dir, args.output_dir)


if __name__ == "__main__":
    main()
