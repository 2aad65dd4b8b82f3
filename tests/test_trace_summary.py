"""tabipb.trace.summarize on a hand-made operation list (host only): the
solve's span, the union of busy intervals (overlapping streams counted once),
per-kernel totals, the LU streams and the idle gaps."""
import re


def test_summary_of_overlapping_streams():
    from tabipb.trace import summarize

    rows = [  # (start_us, end_us, name, stream)
        (0.0, 10.0, "form_matrix_kernel", 7),
        (20.0, 50.0, "lu_np_diag_kernel", 8),     # gap of 10 us before it
        (30.0, 40.0, "near_kernel", 7),          # inside the LU kernel: no gap
        (45.0, 70.0, "lu_gemm2_kernel", 9),      # overlaps the diagonal launch
        (71.0, 80.0, "lu_np_panel_kernel", 8),   # 1 us gap: below the 2 us floor
        (100.0, 101.0, "Memcpy DtoH", 7),        # gap of 20 us
    ]
    out = summarize(rows, top=10, gaps=5)
    span = float(re.search(r"span ([\d.]+) us", out).group(1))
    busy = float(re.search(r"busy \(union\) ([\d.]+) us", out).group(1))
    assert span == 101.0
    # [0, 10] + [20, 70] + [71, 80] + [100, 101]
    assert busy == 10.0 + 50.0 + 9.0 + 1.0
    assert re.search(r"lu_np_diag_kernel\s+1\s+30\.0\s+30\.0", out)
    # two LU streams, with their first start, last end and kernel time
    assert "LU stream 8: 2 launches, 20-80 us, kernel time 39 us" in out
    assert "LU stream 9: 1 launches, 45-70 us, kernel time 25 us" in out
    # the gaps above 2 us: 20 (before the copy) and 10 (before the LU)
    assert "idle gaps > 2 us: 2, 30 us in total" in out
    lines = out.splitlines()
    g = [ln for ln in lines if ln.strip().startswith(("20.0 us", "10.0 us"))]
    assert len(g) == 2 and g[0].strip().startswith("20.0 us")
