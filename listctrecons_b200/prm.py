"""The reference's .prm parameter file: reader and writer.

FileParams follows Src/FileParams.cpp:26-137: whitespace-separated tokens, ``Key:`` followed
by its value, 23 required keys (``TableFeed:`` is an alias of ``PitchValue:``).  The reference
prints the first missing key and calls exit(1) (:18-20); here that is ParameterError with the
same message.  One optional key is new: ``MaxBlocks:`` reconstructs only the first N 32-slice
blocks (the reference has no z-range key; its planner reconstructs every block the table
range allows).
"""
from __future__ import annotations

from dataclasses import dataclass, fields
from pathlib import Path

# Src/FileParams.cpp:10, in the reference's order
TOKEN_NAMES = [
    "RawDataDir", "DataInterpFile", "ViewAngleFile", "CouchPosFile", "OutputDir", "OutputName",
    "Ns", "Nt", "Ds", "Dt", "PitchValue", "Nx", "Ny", "Dx", "Dz", "OffsetX", "OffsetY",
    "Readings", "ViewOffset", "DataOffset", "RSrcToIso", "CentralChannel", "NProjTurn",
]
_INT = {"Ns", "Nt", "Nx", "Ny", "Readings", "ViewOffset", "DataOffset", "NProjTurn"}
_STR = {"RawDataDir", "DataInterpFile", "ViewAngleFile", "CouchPosFile", "OutputDir", "OutputName"}


class ParameterError(ValueError):
    pass


@dataclass
class FileParams:
    RawDataDir: str = ""
    DataInterpFile: str = ""
    ViewAngleFile: str = ""
    CouchPosFile: str = ""
    OutputDir: str = ""
    OutputName: str = ""
    Ns: int = 0
    Nt: int = 0
    Ds: float = 0.0
    Dt: float = 0.0
    PitchValue: float = 0.0
    Nx: int = 0
    Ny: int = 0
    Dx: float = 0.0
    Dz: float = 0.0
    OffsetX: float = 0.0
    OffsetY: float = 0.0
    Readings: int = 0
    ViewOffset: int = 0
    DataOffset: int = 0
    RSrcToIso: float = 0.0
    CentralChannel: float = 0.0
    NProjTurn: int = 0
    MaxBlocks: int = 0  # optional, new

    @classmethod
    def read(cls, path: str | Path) -> "FileParams":
        p = Path(path)
        if not p.is_file():
            raise ParameterError("Parameter file not found. ")
        toks = p.read_text().split()
        have = set()
        fp = cls()
        i = 0
        while i < len(toks):
            t = toks[i]
            key = t[:-1] if t.endswith(":") else None
            if key == "TableFeed":
                key = "PitchValue"
            if key in TOKEN_NAMES or key == "MaxBlocks":
                if i + 1 >= len(toks):
                    break
                raw = toks[i + 1]
                try:
                    val = raw if key in _STR else (int(raw) if key in _INT or key == "MaxBlocks" else float(raw))
                except ValueError as e:
                    raise ParameterError(f"bad value for {key}: {raw!r}") from e
                setattr(fp, key, val)
                have.add(key)
                i += 2
                continue
            i += 1
        for name in TOKEN_NAMES:
            if name not in have:
                raise ParameterError("Parameter not found in prm file:" + name)
        return fp

    def write(self, path: str | Path) -> None:
        lines = []
        for f in fields(self):
            v = getattr(self, f.name)
            if f.name == "MaxBlocks" and not v:
                continue
            if isinstance(v, float):
                lines.append(f"{f.name}: {v!r}")
            else:
                lines.append(f"{f.name}: {v}")
        Path(path).write_text("\n".join(lines) + "\n")

    # accessor names of Include/FileParams.h
    def ns(self): return self.Ns
    def nt(self): return self.Nt
    def ds(self): return self.Ds
    def dt(self): return self.Dt
    def pitch_value(self): return self.PitchValue
    def nx(self): return self.Nx
    def ny(self): return self.Ny
    def dx(self): return self.Dx
    def dz(self): return self.Dz
    def readings(self): return self.Readings
    def r_src_to_iso(self): return self.RSrcToIso
    def central_channel(self): return self.CentralChannel
    def n_proj_turn(self): return self.NProjTurn
