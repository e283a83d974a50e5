"""Roofline of the intra search on B200 (the roofline object of bench.py's JSON line).

The search is integer work (prediction, 4x4 Hadamard SATD, butterfly transforms, quantisation, context-coded rates):
its bound is the INT32 issue rate, not the tensor cores and not HBM (≈6.4 algorithmic bytes per pixel).  The
numerator is the ALGORITHMIC operation count of the workload - the CPU oracle's counters over every unit of work the
search does (oracle/count_ops.py, cost model in oracle/plain_search.cpp) - frozen here per qindex for the 12 MP
image; the denominator is the INT32 instruction rate measured on the device (is_probe_int32).
"""
import os

# oracle/count_ops.py on the 4000x3000 seeded step-edge image (seed 12): ops per pixel (analysis, closed loop)
OPS_PER_PX = {120: (16456.9, 830.3), 60: (18144.3, 984.0), 200: (14254.3, 669.4)}
# algorithmic HBM bytes per pixel (4:2:0 8-bit): source 1.5 + reconstruction 1.5 + levels <= 3 + maps / records 0.4
BYTES_PER_PX = 6.4
# DRAM bytes (read + write) per pixel of one launch, from ncu's dram__bytes_read.sum + dram__bytes_write.sum on a
# 1920x1080 case (profiles/k_recon_1080p.md, profiles/k_analysis_1080p.md); traffic grows with the pixels processed
TRAFFIC_PER_PX = {"k_recon": (12.050432e6 + 1.372928e6) / (1920 * 1080), "k_analysis": (3.105792e6 + 3.166208e6) / (1920 * 1080)}
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _peaks():
    import json
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def report(enc, stage_ms, mp, qindex=120, device=0):
    """The roofline object of bench.py's JSON line: the dominant kernel against the measured INT32 rate."""
    from .isearch import probe_int32
    peak_gops, probe_ms = probe_int32(device)
    ops_a, ops_c = OPS_PER_PX.get(qindex, OPS_PER_PX[120])
    # the analysis stage is four kernels (k_analysis_big, k_analysis, k_analysis_tiny, k_analysis_mid), timed together
    stages = {"k_analysis": (stage_ms["analysis"], ops_a), "k_recon": (stage_ms["recon"], ops_c)}
    name = max(stages, key=lambda k: stages[k][0])
    ms, opx = stages[name]
    achieved = opx * mp * 1e6 / (ms * 1e-3) / 1e9
    hbm_peak, hbm_kind = _peaks()
    total_ms = sum(stage_ms.values())
    hbm_gbs = BYTES_PER_PX * mp * 1e6 / (total_ms * 1e-3) / 1e9
    out = {"bound": "int32", "kernel": name, "achieved": round(achieved, 1), "peak": round(peak_gops, 1), "unit": "Gop/s",
           "frac": round(achieved / peak_gops, 4), "peak_source": "measured (is_probe_int32, %.3f ms)" % probe_ms,
           "traffic": round(TRAFFIC_PER_PX[name] * mp * 1e6), "traffic_source": "ncu on 1920x1080, scaled by pixels",
           "ops_per_px": opx,
           "other_kernel": {k: {"ms": round(v[0], 3), "achieved_gops": round(v[1] * mp * 1e6 / (v[0] * 1e-3) / 1e9, 1),
                                "frac": round(v[1] * mp * 1e6 / (v[0] * 1e-3) / 1e9 / peak_gops, 4)}
                            for k, v in stages.items()},
           "hbm": {"achieved_gbs": round(hbm_gbs, 1), "peak_gbs": hbm_peak, "frac": round(hbm_gbs / hbm_peak, 5),
                   "peak_source": hbm_kind + " (MEASURED_PEAKS.json hbm_gbs)"}}
    return out
