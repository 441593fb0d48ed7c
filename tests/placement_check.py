"""Size-independent checks of a decoded population (test infrastructure).

``check_rows`` replays the placement log of the chosen chromosomes on dense
plates and asserts what every correct decode satisfies, at any size, without
searching for positions itself:

* each gene's machine follows the thresholds (placement.py:118-127; float32
  or float64 comparison as the problem says) and a machine's parts come in
  ascending sequencing key, equal keys in gene order (placement.py:128-131);
  the entries after a machine's last part are empty (-1);
* plates open one at a time (a new plate's index is the number of plates so
  far) and a new plate's part sits at column 0, bottom row L-1, in its best
  rotation (placement.py:66-83);
* every placement lies inside its plate and covers only empty cells, its
  rotation exists, and a part added to an existing plate passes the area
  filter (placement.py:56-59);
* the makespan rebuilt from the log with the build-time model
  (placement.py:86-89, 151-156) equals the decoder's bit for bit, and a
  chromosome scores 1e16 exactly when some part goes to a machine whose plate
  it fits in no orientation (placement.py:47-53, 151-153).

What it does not prove is that each position is the bottom-left-most one and
each plate the first that fits; the oracle checks that on samples.
"""
from __future__ import annotations

from typing import Iterable

import numpy as np

from brkga_fft2_b200 import THRESH_F32

INFEASIBLE = 1e16


class PlacementError(AssertionError):
    pass


def _fail(row: int, m: int, k: int, what: str):
    raise PlacementError(f"row {row}, machine {m}, entry {k}: {what}")


def machine_of(keys: np.ndarray, thresholds: np.ndarray, M: int, mode: int) -> np.ndarray:
    """Machine of each machine key; M for a NaN key (it reaches no machine) unless M == 1."""
    keys = np.asarray(keys, np.float32)
    if M <= 1:
        return np.zeros(keys.shape, np.int64)
    thr = thresholds[: M - 1]
    if mode == THRESH_F32:
        le = keys[..., None] <= thr.astype(np.float32)
    else:
        le = keys.astype(np.float64)[..., None] <= thr.astype(np.float64)
    le = np.concatenate([le, np.ones(keys.shape + (1,), bool)], axis=-1)  # the last machine takes the rest
    m = np.argmax(le, axis=-1)
    return np.where(np.isnan(keys), M, m)


def rotation_masks(packed):
    """Boolean mask of every (part type, rotation) slot, keyed t * 4 + r."""
    a = packed.arrays
    out = {}
    for i, (h, w, off) in enumerate(zip(a["rot_h"], a["rot_w"], a["rot_mask_offset"])):
        out[i] = a["masks"][off: off + h * w].reshape(h, w).astype(bool)
    return out


def check_rows(packed, chromosomes: np.ndarray, makespans: np.ndarray, log: np.ndarray,
               rows: Iterable[int]) -> int:
    """Check the given rows; ``log`` is the structured [P, M, N] placement
    array (gene, bin, x, y, rot).  Returns the number of placements replayed."""
    a = packed.arrays
    N, M = packed.n_genes, packed.n_machines
    T = packed.n_types
    gene_type = a["gene_type"]
    L_of, W_of = a["bin_length"], a["bin_width"]
    pt, pth = a["proc_time"].reshape(M, T), a["proc_time_height"].reshape(M, T)
    rot_h, rot_w = a["rot_h"], a["rot_w"]
    masks = rotation_masks(packed)
    n_placed = 0
    for row in rows:
        ch = np.asarray(chromosomes[row], np.float32)
        seqk, mkey = ch[:N], ch[N:]
        mach = machine_of(mkey, a["thresholds"], M, packed.threshold_mode)
        # placement.py:47-53: a part that fits no orientation of its machine's plate
        t_all = gene_type
        h0, w0 = rot_h[t_all * 4], rot_w[t_all * 4]
        on = mach < M
        Lg = np.where(on, L_of[np.minimum(mach, M - 1)], 0)
        Wg = np.where(on, W_of[np.minimum(mach, M - 1)], 0)
        unfit = on & ((h0 > Lg) | (w0 > Wg)) & ((w0 > Lg) | (h0 > Wg))
        if unfit.any():
            if makespans[row] != INFEASIBLE:
                _fail(row, int(mach[unfit][0]), -1, f"a part fits no orientation of its machine, "
                                                    f"makespan {makespans[row]!r} is not 1e16")
            continue
        if makespans[row] == INFEASIBLE:
            _fail(row, -1, -1, "scored 1e16 although every part fits its machine")
        worst = 0.0
        for m in range(M):
            genes = np.flatnonzero(mach == m)
            k0 = np.where(seqk[genes] == 0.0, np.float32(0.0), seqk[genes])  # -0 == +0
            order = genes[np.lexsort((genes, k0.astype(np.float64)))]
            lg = log[row, m]
            if not (lg["gene"][: order.size] == order).all():
                k = int(np.argmax(lg["gene"][: order.size] != order))
                _fail(row, m, k, f"gene {int(lg['gene'][k])}, expected {int(order[k])} (decode order)")
            if (lg["gene"][order.size:] != -1).any():
                _fail(row, m, order.size, "entries after the machine's last part are not empty")
            L, W = int(L_of[m]), int(W_of[m])
            plates, area, ptb, pthb = [], [], [], []
            for k, g in enumerate(order):
                e = lg[k]
                t = int(gene_type[g])
                r, b, x, y = int(e["rot"]), int(e["bin"]), int(e["x"]), int(e["y"])
                if not 0 <= r < int(a["part_nrot"][t]):
                    _fail(row, m, k, f"rotation {r} of a part with {int(a['part_nrot'][t])}")
                h, w = int(rot_h[t * 4 + r]), int(rot_w[t * 4 + r])
                pa = float(a["part_area"][t])
                if b == len(plates):
                    if (x, y, r) != (0, L - 1, int(a["part_best_rot"][t])):
                        _fail(row, m, k, f"new plate {b} at x={x}, y={y}, rotation {r}")
                    plates.append(np.zeros((L, W), bool))
                    area.append(0.0)
                    ptb.append(0.0)
                    pthb.append(0.0)
                elif not 0 <= b < len(plates):
                    _fail(row, m, k, f"plate {b} with {len(plates)} open")
                elif area[b] + pa > float(a["bin_area"][m]):
                    _fail(row, m, k, f"plate {b} fails the area filter")
                ty = y - h + 1
                if ty < 0 or y > L - 1 or x < 0 or x + w > W:
                    _fail(row, m, k, f"{h}x{w} at x={x}, y={y} leaves the {L}x{W} plate")
                cells = plates[b][ty:y + 1, x:x + w]
                if (cells & masks[t * 4 + r]).any():
                    _fail(row, m, k, f"overlaps a placed part on plate {b} at x={x}, y={y}")
                cells |= masks[t * 4 + r]
                area[b] += pa
                ptb[b] += float(pt[m, t])
                v = float(pth[m, t])
                if v > pthb[b]:
                    pthb[b] = v
                n_placed += 1
            ms = 0.0
            for b in range(len(plates)):
                ms += (ptb[b] + pthb[b]) + float(a["setup_time"][m])
            if ms > worst:
                worst = ms
        if makespans[row] != worst:
            _fail(row, -1, -1, f"makespan {makespans[row]!r}, rebuilt from the log {worst!r}")
    return n_placed
