"""Field comparison helpers shared by the GPU parity tests: per-field error
statistics of a GPU field against an FP64 field (the reference's or the
oracle's), sign flips, and an optional JSON-lines log (TSR_PARITY_LOG)."""
import json
import os

import numpy as np

# FP32 kernel values with FP64 sums against the FP64 reference.  A kernel value
# within FP32 rounding of the EPSILON acceptance threshold (Occupancy.cpp:
# 334-340) can be accepted on one side and not the other, which moves a whole
# term: such leaves are counted, at most OUTLIER_FRAC of them.
KSUM_RTOL = 2e-4
LEN_RTOL = 1e-9
# A prior sums cone lengths over a sphere of 25 leaf sizes, so one threshold
# leaf's length term moves the priors of every leaf whose sphere holds it, by
# at most that term over the sphere's total (measured up to 1.2e-5).  Where
# no cone length differs, the priors are exact (measured error 0).
PRIOR_ATOL = 1e-4
PRIOR_EXACT = 1e-12
OUTLIER_FRAC = 1e-3


def log(record):
    path = os.environ.get("TSR_PARITY_LOG")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(record) + "\n")


def field_stats(ref_fields, gpu, leaves):
    """Max / mean relative error per field and the counts outside tolerance."""
    out = {}
    for name, key, rtol in [("emptiness_sum", "e_sum", KSUM_RTOL), ("sampleness_sum", "s_sum", KSUM_RTOL),
                            ("emptiness_length", "e_len", LEN_RTOL), ("sampleness_length", "s_len", LEN_RTOL)]:
        a, b = gpu.field(name), np.asarray(ref_fields[key])
        err = np.abs(a - b)
        rel = err / np.maximum(np.abs(b), 1e-300)
        out[name] = dict(max_rel=float(rel.max()) if rel.size else 0.0, mean_rel=float(rel.mean()) if rel.size else 0.0,
                         outside=int((err > rtol * np.abs(b) + 1e-12 * np.abs(b).max()).sum()))
    pa, pb = gpu.getPriorForEmptiness(), np.asarray(ref_fields["prior"])
    both = np.isfinite(pa) & np.isfinite(pb)
    d = np.abs(pa[both] - pb[both])
    lengths_equal = out["emptiness_length"]["outside"] == 0 and out["sampleness_length"]["outside"] == 0
    bound = PRIOR_ATOL if not lengths_equal else PRIOR_EXACT
    out["prior_emptiness"] = dict(max_abs=float(d.max()) if d.size else 0.0, mean_abs=float(d.mean()) if d.size else 0.0,
                                  outside=int((d > bound).sum()), bound=bound,
                                  nan_mismatch=int((np.isfinite(pa) != np.isfinite(pb)).sum()))
    oa, ob = gpu.getOccupancy(), np.asarray(ref_fields["occ"])
    flips = np.nonzero((oa > 0) != (ob > 0))[0]
    out["sign_flips"] = [int(x) for x in flips[:50]]
    out["sign_flip_count"] = int(flips.size)
    out["leaves"] = int(leaves)
    cc = float(ref_fields["cone_count"])
    out["cone_count_rel"] = abs(gpu.field("cone_count") - cc) / (abs(cc) if cc != 0.0 else 1.0)
    return out
