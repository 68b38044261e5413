"""STOPTW instances: POIs, the Solomon and Cordeau readers, the simulator's
structure-of-arrays view, and the seeded synthetic-instance generator.

Mirrors the reference's data layer:
  * ``POI`` / ``Instance`` and the two readers follow
    engine/instance.hpp:15-28 (structs), :49-88 (parse_solomon: score = the
    demand column, depot id 0, tmax = the depot's due time) and :90-121
    (parse_cordeau); ``load_instance`` picks the reader by the ``pr`` prefix
    (:129-132).
  * ``SimData`` follows engine/sim_host.hpp:12-40: customers 0..n-1 in id
    order, an (n+1)x(n+1) row-major distance matrix with the depot at index 0,
    each entry ``sqrt(dx*dx + dy*dy)`` evaluated as separate IEEE operations.

The generator (no reference counterpart) writes Solomon-format text, so the
same bytes feed this reader, the reference reader and every evaluator.
"""
from __future__ import annotations

import math
import random
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np


@dataclass
class POI:
    id: int
    x: float
    y: float
    score: float
    open_time: float
    close_time: float
    duration: float


@dataclass
class Instance:
    name: str
    pois: List[POI]  # sorted by id; pois[0] is the depot
    tmax: float
    source: str = ""

    @property
    def n_customers(self) -> int:
        return len(self.pois) - 1


def _starts_with_digit(tok: str) -> bool:
    t = tok.lstrip("-")
    return bool(t) and all("0" <= c <= "9" for c in t)


def parse_solomon_text(text: str, source: str = "") -> Instance:
    """engine/instance.hpp:49-88."""
    lines = [ln.strip(" \t\r\n") for ln in text.splitlines()]
    lines = [ln for ln in lines if ln]
    name = lines[0].lower()
    cust = 0
    for i, ln in enumerate(lines):
        if "CUST" in ln.upper():
            cust = i
            break
    pois = []
    for ln in lines[cust + 1:]:
        parts = ln.split()
        if len(parts) < 7 or not _starts_with_digit(parts[0]):
            continue
        pid = int(parts[0])
        demand = float(parts[3])
        pois.append(POI(pid, float(parts[1]), float(parts[2]), 0.0 if pid == 0 else demand,
                        float(parts[4]), float(parts[5]), float(parts[6])))
    pois.sort(key=lambda p: p.id)
    return Instance(name, pois, pois[0].close_time, source)


def parse_cordeau_text(text: str, stem: str, source: str = "") -> Instance:
    """engine/instance.hpp:90-121."""
    pois = []
    for ln in text.splitlines():
        parts = ln.split()
        if len(parts) < 9 or not _starts_with_digit(parts[0]):
            continue
        cid = int(parts[0])
        if cid < 0:
            continue
        pois.append(POI(cid, float(parts[1]), float(parts[2]),
                        0.0 if cid == 0 else float(parts[4]),
                        float(parts[-2]), float(parts[-1]), float(parts[3])))
    pois.sort(key=lambda p: p.id)
    return Instance(stem.lower(), pois, pois[0].close_time, source)


def load_instance_file(path: str) -> Instance:
    """load_instance by file path: Cordeau for ``pr*`` stems, else Solomon."""
    import os
    stem = os.path.splitext(os.path.basename(path))[0]
    with open(path) as f:
        text = f.read()
    if stem.startswith("pr"):
        return parse_cordeau_text(text, stem, path)
    return parse_solomon_text(text, path)


@dataclass
class SimData:
    """The evaluator's view of one instance (engine/sim_host.hpp:12-40)."""
    n: int
    m: int
    tmax: float
    scores: np.ndarray
    durations: np.ndarray
    open_t: np.ndarray
    close_t: np.ndarray
    dist: np.ndarray  # (n+1)*(n+1), row-major, depot = 0
    dist_to_depot: np.ndarray
    sigma: float = 0.2
    name: str = ""
    coords: Optional[np.ndarray] = field(default=None, repr=False)

    @property
    def ld(self) -> int:
        return self.n + 1

    @staticmethod
    def from_instance(inst: Instance, m: int = 3, sigma: float = 0.2) -> "SimData":
        P = inst.pois
        return SimData.from_arrays(
            [p.x for p in P], [p.y for p in P], [p.score for p in P],
            [p.open_time for p in P], [p.close_time for p in P], [p.duration for p in P],
            inst.tmax, m=m, sigma=sigma, name=inst.name)

    @staticmethod
    def from_arrays(x, y, score, open_t, close_t, duration, tmax, m: int = 3,
                    sigma: float = 0.2, name: str = "") -> "SimData":
        """POI arrays in id order, index 0 = depot."""
        x = np.asarray(x, dtype=np.float64)
        y = np.asarray(y, dtype=np.float64)
        dx = x[:, None] - x[None, :]
        dy = y[:, None] - y[None, :]
        dist = np.sqrt(dx * dx + dy * dy)  # separate IEEE mul/mul/add/sqrt
        return SimData(
            n=len(x) - 1, m=m, tmax=float(np.asarray(tmax).reshape(-1)[0]),
            scores=np.ascontiguousarray(np.asarray(score, dtype=np.float64)[1:]),
            durations=np.ascontiguousarray(np.asarray(duration, dtype=np.float64)[1:]),
            open_t=np.ascontiguousarray(np.asarray(open_t, dtype=np.float64)[1:]),
            close_t=np.ascontiguousarray(np.asarray(close_t, dtype=np.float64)[1:]),
            dist=np.ascontiguousarray(dist.reshape(-1)),
            dist_to_depot=np.ascontiguousarray(dist[1:, 0]),
            sigma=sigma, name=name, coords=np.stack([x, y], axis=1))


# ---------------------------------------------------------------- generator

def _fmt(v: float) -> str:
    return repr(float(v)) if v != int(v) else str(int(v))


def solomon_text(name: str, m: int, rows) -> str:
    """Solomon-format text: ``CUST`` header, then ``id x y demand ready due service``."""
    out = [name.upper(), "", "VEHICLE", "NUMBER     CAPACITY", f"  {m}         200", "",
           "CUSTOMER",
           "CUST NO.  XCOORD.   YCOORD.    DEMAND   READY TIME  DUE DATE   SERVICE   TIME", ""]
    for r in rows:
        out.append("  ".join(_fmt(v) for v in r))
    return "\n".join(out) + "\n"


def generate_instance(n: int, layout: str, horizon: float, seed: int, n_clusters: int = 8,
                      service: float = 10.0, name: Optional[str] = None):
    """Seeded synthetic STOPTW instance, returned as Solomon text.

    layout: ``uniform`` (integer coordinates uniform on [0,100]^2), ``clustered``
    (``n_clusters`` Gaussian centres uniform on [0,100]^2, sigma 5, rounded and
    clipped to [0,100]) or ``mixed`` (half of each).  The depot sits at (50,50)
    with window [0, horizon].  Scores are integers uniform in 1..50, service
    time ``service``; each window is centred at an integer drawn uniformly in
    [ceil(d0i), floor(horizon - service - d0i)] with an integer half-width
    uniform in 5..60, clipped to [0, horizon].
    """
    rng = random.Random(seed)
    centres = [(rng.uniform(0, 100), rng.uniform(0, 100)) for _ in range(n_clusters)]
    rows = [(0, 50, 50, 0, 0, int(horizon) if horizon == int(horizon) else horizon, 0)]
    for i in range(1, n + 1):
        use_cluster = layout == "clustered" or (layout == "mixed" and i % 2 == 0)
        if use_cluster:
            cx, cy = centres[rng.randrange(n_clusters)]
            x = min(100, max(0, int(round(rng.gauss(cx, 5.0)))))
            y = min(100, max(0, int(round(rng.gauss(cy, 5.0)))))
        else:
            x = rng.randint(0, 100)
            y = rng.randint(0, 100)
        score = rng.randint(1, 50)
        d0 = math.sqrt((x - 50) ** 2 + (y - 50) ** 2)
        lo = math.ceil(d0)
        hi = math.floor(horizon - service - d0)
        if hi < lo:
            hi = lo
        centre = rng.randint(lo, hi)
        hw = rng.randint(5, 60)
        ready = max(0, centre - hw)
        due = min(horizon, centre + hw)
        rows.append((i, x, y, score, ready, due, service))
    return solomon_text(name or f"syn_{layout}_{n}_{seed}", 25, rows)
