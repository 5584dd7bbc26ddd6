"""Recursive comparison of diagnostics results with the reference's (JSON)."""

import math


def assert_same(got, want, path="", rtol=1e-9, atol=1e-12):
    if isinstance(want, dict):
        assert isinstance(got, dict), (path, got)
        assert set(got) == set(want), (path, sorted(set(got) ^ set(want)))
        for k in want:
            assert_same(got[k], want[k], f"{path}.{k}", rtol, atol)
    elif isinstance(want, list):
        assert isinstance(got, (list, tuple)) and len(got) == len(want), (path, got, want)
        for i, (g, w) in enumerate(zip(got, want)):
            assert_same(g, w, f"{path}[{i}]", rtol, atol)
    elif isinstance(want, bool) or want is None or isinstance(want, str):
        if isinstance(want, str) and ":" in want and ";" in want:  # "x:value;..." flux samples
            gp = [p.split(":") for p in got.split(";")]
            wp = [p.split(":") for p in want.split(";")]
            assert [a for a, _ in gp] == [a for a, _ in wp], (path, got, want)
            for (_, g), (_, w) in zip(gp, wp):
                assert_same(float(g), float(w), path, max(rtol, 1e-11), atol)
        else:
            assert got == want, (path, got, want)
    elif isinstance(want, int):
        assert got == want and not isinstance(got, bool), (path, got, want)
    else:
        g, w = float(got), float(want)
        if math.isnan(w):
            assert math.isnan(g), (path, g, w)
        else:
            assert g == w or abs(g - w) <= atol + rtol * abs(w), (path, g, w)
