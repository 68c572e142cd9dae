"""The reference's data.dat reader and Config mapping, restated for the host side.

read_data_dat  follows ReadInputFile (FREHD.c:30-63): '#' lines are skipped,
               everything after the first ';' is ignored, the first four
               entries are strings, the rest are parsed with strtod.
config_from_values follows ReadUserSettings (configuration.c:18-159) for the
               fields the step reads, including its integer truncations.
"""
from __future__ import annotations

FIELDS = [
    "nx", "ny", "dx", "dy", "dt", "g", "NUx", "NUy", "Kx", "Ky", "CDx", "CDy", "manningN",
    "CDmax", "hD", "CwT", "CDnotN", "useThinLayer", "useSubgrid", "useSubDrag", "staggeredV",
    "useminA", "useminV", "dxf", "dyf", "subR", "surfmin", "surfmax", "dsurf", "bcType",
    "tideLocFirstP", "tideLocLengthP", "useScalar", "scalarAdv", "useConstTidePS", "tidePS",
    "useWind", "useEvap", "useRain", "inflowLocLength", "useSubStep", "checkConservation",
    "minDepth", "wtfh", "CFLl", "CFLh", "eps", "maxIter", "offset",
    "inflowI0", "inflowI1", "inflowJ0", "inflowJ1", "inflowS", "northAngle", "rhoa", "Cw",
    "nscalar",
]


def _strtod(tok: str) -> float:
    tok = tok.strip()
    # strtod reads the longest valid prefix; data.dat entries are plain numbers
    for end in range(len(tok), 0, -1):
        try:
            return float(tok[:end])
        except ValueError:
            continue
    return 0.0


def read_data_dat(path: str) -> list:
    """Positional values of a data.dat (FREHD.c:30-63)."""
    vals = []
    with open(path) as f:
        for line in f:
            if line.startswith("#"):
                continue
            tok = line.split(";", 1)[0]
            if len(vals) < 4:
                vals.append(tok)
            else:
                vals.append(_strtod(tok))
    return vals


def config_from_values(v: list, offset: float = 0.0) -> dict:
    """Config fields of ReadUserSettings (configuration.c:23-127) from data.dat values."""
    i = int
    dx, dy = float(v[4]), float(v[5])
    NX, NY = i(v[6]), i(v[7])
    np_ = i(v[66])
    dxf, dyf = float(v[56]), float(v[57])
    c = dict(
        nx=NX, ny=i(round(NY / np_)) if np_ else NY, dx=dx, dy=dy, dt=float(v[8]),
        bcType=i(v[19]), tideLocLengthP=i(v[20]), tideLocFirstP=i(v[21]),
        useWind=i(v[32]), useScalar=i(v[36]), scalarAdv=i(v[37]),
        useConstTidePS=i(v[40]), tidePS=float(v[41]),
        useSubgrid=i(v[54]), useSubDrag=i(v[55]), dxf=dxf, dyf=dyf, subR=dx / dxf,
        surfmax=float(v[58]), surfmin=float(v[59]), dsurf=float(v[60]),
        staggeredV=i(v[61]), useminA=i(v[62]), useminV=i(v[64]),
        g=float(v[67]), NUx=float(v[68]), NUy=float(v[69]), CDnotN=i(v[70]),
        CDx=float(v[71]), CDy=float(v[72]), manningN=float(v[73]), useThinLayer=i(v[74]),
        hD=float(v[75]), CDmax=float(v[76]), CwT=float(v[77]), Kx=float(v[80]),
        Ky=float(v[81]), minDepth=float(v[82]), wtfh=float(v[83]), CFLl=float(v[84]),
        CFLh=float(v[85]), eps=float(v[86]), maxIter=i(v[87]),
        # never assigned by ReadUserSettings; zero under a zeroing allocator
        useEvap=0, useRain=0, useSubStep=0, checkConservation=0,
        inflowLocLength=i(v[26]), offset=offset,
        # inflowLoc[k] = jj*NX + ii - 1 for ii in [v27, v28), jj in [v29, v30)
        # (configuration.c:53-60): cells i in [v27 - 1, v28 - 1), j in [v29, v30)
        inflowI0=i(v[27]) - 1, inflowI1=i(v[28]) - 1, inflowJ0=i(v[29]), inflowJ1=i(v[30]),
        inflowS=float(v[39]), northAngle=float(v[33]), rhoa=float(v[78]), Cw=float(v[79]),
        nscalar=1,  # the reference carries one scalar, S
    )
    return c


def n_levels(c: dict) -> int:
    """Ne = round((surfmax - surfmin)/dsurf) (subgrid.c:2115)."""
    return int(round((c["surfmax"] - c["surfmin"]) / c["dsurf"]))


def fill_struct(struct, c: dict):
    for k in FIELDS:
        setattr(struct, k, c[k])
    return struct
