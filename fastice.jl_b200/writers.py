"""Field output and checkpoints: the reference's Writers module (src/Writers.jl)
and a resumable dump of a PT solve.

* ``write_xdmf(grid, path, fields, h5_names, timesteps=0.0)`` -- Xdmf 3 metadata
  of Center fields, element for element and number for number as
  ``generate_xdmf`` / ``create_xdmf_attribute`` (Writers.jl:80-137) write it: a
  temporal collection of uniform grids (3DCoRectMesh topology with the vertex
  counts, ORIGIN_DXDYDZ geometry with the first cell centre and the spacing, in
  z, y, x order) with one Cell attribute per field pointing into ``<file>.h5:/<name>``.
  ``data_format="binary"`` points the attributes at raw files instead (what
  ``write_raw`` writes), which Xdmf readers open without HDF5.
* ``write_h5(grid, path, fields)`` -- the datasets ``/<name>`` of ``write_h5`` /
  ``write_dset`` (Writers.jl:19-58), through h5py when it is installed (this
  image has no HDF5 library; the call then raises FastIceError).
* ``write_raw(path, fields)`` -- each field's interior as little-endian raw data,
  x fastest (the Julia column-major order of ``Array(interior(field))``).
* ``save_checkpoint(model, directory)`` / ``load_checkpoint(model, directory)`` --
  the PT state (P, τ, V, η) as raw little-endian dumps plus a JSON sidecar (grid,
  dtype, shapes); loading sets the fields and re-applies the boundary
  conditions, so a solve continues where it stopped.

Floats print as Julia prints a Float64 (shortest round trip; exponent form
``1.0e-5``), so the metadata matches the reference's text.
"""
from __future__ import annotations

import json
import os
from typing import Iterable, Mapping, Sequence, Union

import numpy as np

from . import _lib as L


def julia_float(x: float) -> str:
    """``string(x::Float64)`` in Julia: the shortest round-trip digits; the
    exponent form writes ``1.0e-5`` where Python writes ``1e-05``."""
    s = repr(float(x))
    if s in ("inf", "-inf", "nan"):
        return {"inf": "Inf", "-inf": "-Inf", "nan": "NaN"}[s]
    if "e" in s:
        mant, exp = s.split("e")
        if "." not in mant:
            mant += ".0"
        return f"{mant}e{int(exp)}"
    return s


def _names(fields) -> list:
    return list(fields.keys()) if isinstance(fields, Mapping) else list(fields)


def _attribute_lines(ind: str, name: str, dims: str, source: str, data_format: str, esz: int) -> list:
    if data_format == "hdf":
        item = (f'<DataItem Format="HDF" NumberType="Float" Precision="8" Dimensions="{dims}">'
                f"{source}:/{name}</DataItem>")
    else:
        item = (f'<DataItem Format="Binary" NumberType="Float" Precision="{esz}" Endian="Little" '
                f'Dimensions="{dims}">{source}</DataItem>')
    return [f'{ind}<Attribute Name="{name}" Center="Cell">', f"{ind}  {item}", f"{ind}</Attribute>"]


def xdmf_text(grid, fields, h5_names: Sequence[str], timesteps: Union[float, Iterable[float]] = 0.0,
              data_format: str = "hdf", raw_names=None, precision: int = 8) -> str:
    """The Xdmf document write_xdmf writes (Writers.jl:80-137)."""
    ts = [float(timesteps)] if np.isscalar(timesteps) else [float(t) for t in timesteps]
    names = _names(fields)
    size = tuple(grid.dims)
    spacing = tuple(grid.spacing())
    origin_c = tuple(o + d / 2 for o, d in zip(grid.origin, spacing))
    rev = lambda t: " ".join(str(v) for v in reversed(t))  # noqa: E731
    out = ['<?xml version="1.0" encoding="utf-8"?>', '<Xdmf Version="3.0">', "  <Domain>",
           '    <Grid GridType="Collection" CollectionType="Temporal">']
    for it, tt in enumerate(ts):
        h5 = h5_names[it]
        if data_format == "hdf" and not h5.endswith(".h5"):
            raise ValueError("h5 file names must end in .h5")
        out += ['      <Grid GridType="Uniform">',
                f'        <Topology TopologyType="3DCoRectMesh" Dimensions="{rev(tuple(n + 1 for n in size))}"/>',
                f'        <Time Value="{julia_float(tt)}"/>',
                '        <Geometry GeometryType="ORIGIN_DXDYDZ">',
                f'          <DataItem Format="XML" NumberType="Float" Dimensions="{len(size)}">'
                f'{" ".join(julia_float(v) for v in reversed(origin_c))}</DataItem>',
                f'          <DataItem Format="XML" NumberType="Float" Dimensions="{len(size)}">'
                f'{" ".join(julia_float(v) for v in reversed(spacing))}</DataItem>',
                "        </Geometry>"]
        for k, name in enumerate(names):
            src = h5 if data_format == "hdf" else raw_names[it][k]
            out += _attribute_lines("        ", name, rev(size), src, data_format, precision)
        out.append("      </Grid>")
    out += ["    </Grid>", "  </Domain>", "</Xdmf>"]
    return "\n".join(out) + "\n"


def write_xdmf(grid, path: str, fields, h5_names: Sequence[str], timesteps: Union[float, Iterable[float]] = 0.0,
               data_format: str = "hdf", raw_names=None, precision: int = 8) -> None:
    """``write_xdmf(arch, grid, path, fields, h5_names, timesteps)`` (Writers.jl:65-71).
    ``fields``: names (or a mapping whose keys are the names), in output order.
    ``data_format="binary"``: ``raw_names[t][k]`` is the raw file of field k at time
    step t (``write_raw``'s output), precision the bytes per value."""
    with open(path, "w", encoding="utf-8") as f:
        f.write(xdmf_text(grid, fields, h5_names, timesteps, data_format, raw_names, precision))


def write_h5(grid, path: str, fields: Mapping[str, np.ndarray]) -> None:
    """``write_h5(arch, grid, path, fields)`` (Writers.jl:19-25): one dataset per
    field with the interior values (h5py's C order (z, y, x) is the file layout
    Julia's column-major (x, y, z) writes).  Needs h5py."""
    try:
        import h5py
    except ImportError as e:
        raise L.FastIceError(L.FI_ERR_UNSUPPORTED, "write_h5 needs h5py (no HDF5 library is installed); "
                                                   "write_raw + write_xdmf(data_format='binary') "
                                                   "write the same data without it") from e
    with h5py.File(path, "w") as f:
        for name, arr in fields.items():
            a = np.asarray(arr)
            if a.shape != tuple(reversed(grid.dims)):
                raise ValueError(f"{name}: a Center field of the grid has shape {tuple(reversed(grid.dims))}")
            f.create_dataset(name, data=a)


def write_raw(path: str, fields: Mapping[str, np.ndarray]) -> dict:
    """Each field's interior as little-endian raw values, x fastest, to
    ``<path>.<name>.raw``; returns {name: file name}."""
    out = {}
    for name, arr in fields.items():
        a = np.asarray(arr)
        fn = f"{path}.{name}.raw"
        a.astype(a.dtype.newbyteorder("<"), copy=False).tofile(fn)
        out[name] = fn
    return out


STATE_FIELDS_3D = ("P", "txx", "tyy", "tzz", "txy", "txz", "tyz", "Vx", "Vy", "Vz", "eta")
STATE_FIELDS_2D = ("P", "txx", "tyy", "txy", "Vx", "Vy", "eta")


def save_checkpoint(model, directory: str) -> None:
    """The PT state of ``model`` (P, τ, V, η interiors) as raw little-endian dumps
    plus ``checkpoint.json`` (grid, dtype, shapes)."""
    os.makedirs(directory, exist_ok=True)
    nd = model.grid.ndims
    names = STATE_FIELDS_3D if nd == 3 else STATE_FIELDS_2D
    meta = {"dims": list(model.grid.dims), "origin": list(model.grid.origin), "extent": list(model.grid.extent),
            "dtype": model.dtype, "fields": {}}
    for name in names:
        a = model.get_field(name)
        fn = f"{name}.raw"
        a.astype(a.dtype.newbyteorder("<"), copy=False).tofile(os.path.join(directory, fn))
        meta["fields"][name] = {"file": fn, "shape": list(a.shape)}
    with open(os.path.join(directory, "checkpoint.json"), "w") as f:
        json.dump(meta, f, indent=1)


def load_checkpoint(model, directory: str) -> dict:
    """Restore a state written by ``save_checkpoint`` into a model of the same grid
    and dtype: sets every field (η_next = η) and re-applies the boundary
    conditions; returns the sidecar."""
    with open(os.path.join(directory, "checkpoint.json")) as f:
        meta = json.load(f)
    if list(model.grid.dims) != meta["dims"] or model.dtype != meta["dtype"]:
        raise ValueError("the checkpoint was written for another grid or dtype")
    npd = np.float64 if meta["dtype"] == "f64" else np.float32
    for name, d in meta["fields"].items():
        a = np.fromfile(os.path.join(directory, d["file"]), dtype=np.dtype(npd).newbyteorder("<"))
        model.set_field(name, a.reshape(d["shape"]).astype(npd))
        if name == "eta":
            model.set_field("eta_next", a.reshape(d["shape"]).astype(npd))
    model.apply_bcs()
    return meta


__all__ = ["julia_float", "xdmf_text", "write_xdmf", "write_h5", "write_raw", "save_checkpoint", "load_checkpoint"]
