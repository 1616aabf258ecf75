"""The autotuner's partial re-tune (--only) on the CPU: entries of the load
balances that were re-tuned come from the new run, every other entry, shape
and report line from the earlier table."""
import numpy as np

import gswitch_b200 as gs
from gswitch_b200.autotune import VARIANTS, merge, shapes_of


def test_only_replaces_the_retuned_load_balances():
    old_q = np.arange(gs.TUNE_ENTRIES, dtype=np.int32) % 7 + 1
    old_s = np.zeros(gs.TUNE_ENTRIES, dtype=np.int32)
    old_s[gs.Context.tune_index("Push", "Queue", "STRICT")] = 2
    old = {"quarters": [int(x) for x in old_q], "shapes": [int(x) for x in old_s],
           "report": {"Push-Queue-STRICT-Standalone": {"shape": 2}, "Pull-Bitmap-TM-Standalone": {"shape": 0}}}
    new_q = np.zeros(gs.TUNE_ENTRIES, dtype=np.int32)
    new_s = np.zeros(gs.TUNE_ENTRIES, dtype=np.int32)
    tm = gs.Context.tune_index("Pull", "Bitmap", "TM")
    new_q[tm], new_s[tm] = 16, 4
    q, s, rep = merge(old, new_q, new_s, {"Pull-Bitmap-TM-Standalone": {"shape": 4}}, {"TM"})
    for d, f, lb, fused in VARIANTS:
        i = gs.Context.tune_index(d, f, lb, fused)
        if lb == "TM":
            assert (q[i], s[i]) == (new_q[i], new_s[i])
        else:
            assert (q[i], s[i]) == (old_q[i], old_s[i])
    assert rep == {"Push-Queue-STRICT-Standalone": {"shape": 2}, "Pull-Bitmap-TM-Standalone": {"shape": 4}}
    assert not np.shares_memory(q, new_q)


def test_shape_counts_match_the_library():
    assert shapes_of("Pull", "TM") == 9 and shapes_of("Push", "TM") == 3
    assert shapes_of("Push", "STRICT") == shapes_of("Pull", "STRICT") == 3
    assert shapes_of("Push", "WM") == shapes_of("Pull", "TWC") == 1
