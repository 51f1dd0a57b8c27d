"""Per-shape tuning of the DFT stage tile width, cached to JSON.

The tcgen05 stage kernel computes output tiles of 128 rows x N_TILE real
columns; with the 3-term BF16 split N_TILE may be 64, 128 or 256.  A short
output axis wastes most of a wide tile (the forward stage of a 32-sample
axis fills 64 of 256 columns), while narrow tiles stage every operand row
once more per extra column tile.  Which wins depends on the shape and on
how many scenes share the GPU, so the tuner times one solve per candidate
width on the device and keeps the fastest.

Results are cached per (N1, N2, M1, M2, terms, batch class, device name)
in a JSON file: ``$FBME_B200_AUTOTUNE_CACHE`` or
``~/.cache/fbme_b200/autotune.json``.  The batch class is the batch size
rounded up to a power of two.
"""

from __future__ import annotations

import json
import os
import tempfile
from math import ceil, prod
from pathlib import Path
from typing import Callable, Sequence

CACHE_ENV = "FBME_B200_AUTOTUNE_CACHE"
TILE_ROWS = 128            # rows of a stage tile (the UMMA M)
MAX_TILES_PER_SCENE = 64   # partial-sum slots per scene and stage

Shape = tuple[tuple[int, int], tuple[int, int]]


def default_cache_path() -> Path:
    env = os.environ.get(CACHE_ENV)
    if env:
        return Path(env)
    return Path.home() / ".cache" / "fbme_b200" / "autotune.json"


def candidates(grid: Sequence[int], sample: Sequence[int], terms: int = 3) -> list[int]:
    """Tile widths the library accepts for this shape: 64, 128, 256 with 3
    terms (128 with 6), at most 64 tiles per scene in each of the four
    stages (rows x columns: N1 x M2, M2 x M1, M1 x N2, N2 x N1)."""
    n1, n2 = (int(v) for v in grid)
    m1, m2 = (int(v) for v in sample)
    widths = (128,) if terms == 6 else (64, 128, 256)
    stages = ((n1, m2), (m2, m1), (m1, n2), (n2, n1))
    return [w for w in widths
            if all(ceil(r / TILE_ROWS) * ceil(2 * c / w) <= MAX_TILES_PER_SCENE for r, c in stages)]


def stage_tiles(grid: Sequence[int], sample: Sequence[int], width: int) -> list[int]:
    """Tiles of one scene in each of the four DFT stages at a tile width."""
    n1, n2 = (int(v) for v in grid)
    m1, m2 = (int(v) for v in sample)
    return [ceil(r / TILE_ROWS) * ceil(2 * c / width) for r, c in ((n1, m2), (m2, m1), (m1, n2), (n2, n1))]


def default_width(grid: Sequence[int], sample: Sequence[int], batch: int, terms: int = 3, sms: int = 148) -> int:
    """Tile width when none is given or cached.  Once the batch's stage
    tiles at the widest width outnumber the SMs, the widest width (fewest
    operand re-reads) wins; below that the narrowest allowed width, whose
    extra tiles keep more SMs busy.  Measured on B200 (Stable, 256x256 /
    128x128): one scene solves in 0.56 ms with 64-column tiles against
    0.64 ms with 256; 64 and 256 scenes are fastest with 256 columns."""
    cands = candidates(grid, sample, terms)
    if terms == 6 or not cands:
        return 128 if terms == 6 else 256
    widest = max(cands)
    if batch * sum(stage_tiles(grid, sample, widest)) >= sms:
        return widest
    return min(cands)


def batch_class(batch: int) -> int:
    b = 1
    while b < batch and b < 4096:
        b *= 2
    return b


def cache_key(grid: Sequence[int], sample: Sequence[int], terms: int, batch: int, device_name: str) -> str:
    n1, n2 = grid
    m1, m2 = sample
    return f"{n1}x{n2}/{m1}x{m2}/t{terms}/b{batch_class(batch)}/{device_name}"


class TileCache:
    """The JSON cache: {key: {"dft_n_tile": w, "ms": {w: ms}, "batch": b}}."""

    def __init__(self, path: Path | str | None = None) -> None:
        self.path = Path(path) if path is not None else default_cache_path()
        self.entries: dict[str, dict] = {}
        if self.path.exists():
            try:
                self.entries = json.loads(self.path.read_text())
            except (OSError, ValueError):
                self.entries = {}

    def get(self, key: str) -> dict | None:
        return self.entries.get(key)

    def put(self, key: str, entry: dict) -> None:
        self.entries[key] = entry

    def save(self) -> None:
        """Write atomically (a temporary file renamed over the cache)."""
        self.path.parent.mkdir(parents=True, exist_ok=True)
        fd, tmp = tempfile.mkstemp(dir=self.path.parent, prefix=".autotune", suffix=".json")
        with os.fdopen(fd, "w") as f:
            json.dump(self.entries, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)


Timer = Callable[[Sequence[int], Sequence[int], object, object, int, int], float]


def measure(grid: Sequence[int], sample: Sequence[int], cfg, device, batch: int, n_tile: int,
            reps: int = 5) -> float:
    """Device milliseconds of one solve of `batch` synthetic scenes with
    stage tiles `n_tile` wide (CUDA events, after two warm-up solves)."""
    import torch

    import dataclasses

    from .engine import FBMEEngine, resolve_dft_terms

    # timed as the uneven plans run it: the tensor-core stages
    cfg = dataclasses.replace(cfg, dft_terms=resolve_dft_terms(int(cfg.dft_terms), grid, uneven=True))
    eng = FBMEEngine(batch, grid, sample, cfg, device, n_tile=n_tile)
    try:
        g = torch.Generator(device=device).manual_seed(1234)
        y = torch.randn(batch, prod(sample), dtype=torch.complex64, device=device, generator=g)
        for _ in range(2):
            eng.run(y)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        start.record()
        for _ in range(reps):
            eng.run(y)
        stop.record()
        torch.cuda.synchronize(device)
        return start.elapsed_time(stop) / reps
    finally:
        eng.close()


def tune_shape(grid: Sequence[int], sample: Sequence[int], cfg, device, batch: int, *,
               cache: TileCache | None = None, timer: Timer = measure, force: bool = False,
               device_name: str | None = None) -> int:
    """The fastest tile width for this shape and batch class, from the cache
    or measured (and then stored)."""
    from .engine import resolve_dft_terms

    # the tile width of the tensor-core stages, which uneven plans run
    terms = resolve_dft_terms(int(getattr(cfg, "dft_terms", 3)), grid, uneven=True)
    if terms == 0:
        return 256  # the FP32 FFT stages have no tile width to choose
    if device_name is None:
        import torch

        device_name = torch.cuda.get_device_name(device).replace(" ", "_")
    cache = cache if cache is not None else TileCache()
    key = cache_key(tuple(grid), tuple(sample), terms, batch, device_name)
    hit = cache.get(key)
    cands = candidates(grid, sample, terms)
    if hit is not None and not force and hit.get("dft_n_tile") in cands:
        return int(hit["dft_n_tile"])
    times = {w: float(timer(grid, sample, cfg, device, batch, w)) for w in cands}
    best = min(times, key=times.get)
    cache.put(key, {"dft_n_tile": best, "ms": {str(w): t for w, t in times.items()}, "batch": batch})
    cache.save()
    return best


def tune_shapes(shapes: Sequence[Shape], cfg, device, *, cache: TileCache | None = None,
                timer: Timer = measure, force: bool = False,
                device_name: str | None = None) -> dict[Shape, int]:
    """tune_shape for every distinct shape of a scene list, each at the
    number of scenes of that shape."""
    counts: dict[Shape, int] = {}
    for grid, sample in shapes:
        key = (tuple(grid), tuple(sample))
        counts[key] = counts.get(key, 0) + 1
    cache = cache if cache is not None else TileCache()
    return {k: tune_shape(k[0], k[1], cfg, device, n, cache=cache, timer=timer, force=force,
                          device_name=device_name)
            for k, n in counts.items()}
