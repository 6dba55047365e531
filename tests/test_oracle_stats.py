"""The oracle's EncodeFrameStats are consistent with its own side info (CPU)."""
import numpy as np

from oracle import oracle as O


def test_oracle_stats_agree_with_side_info():
    from riv2_b200.synth import SynthClip
    w, h = 352, 288
    clip = SynthClip("cif", seed=81)
    oc = O.default_config(w, h, 30)
    oc.intra_quality, oc.inter_quality = 85, 80
    oc.keyframe_mode, oc.keyframe_interval = 2, 1 << 40
    oe = O.OracleEncoder(oc)
    n = (w // 16) * (h // 16)
    for t in range(4):
        assert oe.encode_rgb(clip.frame(t), t * 33) == 0
        s = oe.last_stats()
        if t == 0:
            assert s["frame_type"] == 1 and s["resi_raw"] is None and s["mv_bytes"] == 0
            continue
        side = oe.last_side()  # mode, base, delta x, delta y, flags, rdo skip, optimized skip, filter
        modes = np.bincount(side[:, 0], minlength=7)
        assert s["mv_mode_counts"] == tuple(float(x) for x in modes)
        assert s["blocks_total"] == n and s["rdo_blocks_evaluated"] == n and s["mv_candidate_unique_samples"] == n
        assert s["mv_new_blocks"] == modes[5] == s["mv_new_delta_count"] == sum(s["mv_new_best_ref_counts"])
        assert s["rdo_blocks_selected_skip"] == side[:, 5].sum()
        assert s["blocks_skipped"] == side[:, 6].sum()
        assert s["resi_raw"] == (n - side[:, 6].sum()) * 768
        assert s["mv_raw_bytes"] == 2 * n + 2 * modes[5]
        assert sum(s["mv_class_histogram"]) == 2 * modes[5]
        assert sum(s["mv_match_source_counts"]) == s["mv_match_nonzero_blocks"]
        assert 1 <= s["mv_candidate_unique_min"] <= s["mv_candidate_unique_max"] <= 5
        assert (s["mv_bias_dx"], s["mv_bias_dy"]) == oe.last_bias()
