"""Post-processing of the solver's output files (the reference's post/ layer).

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


def main() -> None:
    ap = argparse.ArgumentParser(description="Convert mean_profiles/uy_avg.bin to profiles/uy_avg.vti.")
    ap.add_argument("--case-dir", required=True, help="case directory, e.g. JET_VTK/Re120_We8")
    ap.add_argument("--output-dir", default=None, help="defaults to <case-dir>/profiles")
    args = ap.parse_args()
    write_uy_avg_vti(args.case_dir, args.output_dir)


if __name__ == "__main__":
    main()
