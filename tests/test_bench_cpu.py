"""Host logic of bench.py that needs no GPU: the element-kernel name of the
variant the engine reports, and the DRAM traffic looked up from the
committed ncu summary of exactly that variant."""
import os

import bench


class _FakeDC:
    def __init__(self, chosen):
        self.chosen = chosen

    def element_variants(self):
        return {"chosen": self.chosen, "count": len(bench.ELEMENT_KERNELS_N4)}


def test_element_kernel_name_follows_the_engine_variant():
    for v, name in enumerate(bench.ELEMENT_KERNELS_N4):
        assert bench.element_kernel_name(_FakeDC(v)) == name
    assert bench.element_kernel_name(_FakeDC(-1)) == "k_element<5>"


def _summary(path, title, traffic):
    with open(path, "w") as f:
        f.write(f"# {title} — curved_lake, N=4, 512x512\n\nsome text\n")
        if traffic is not None:
            f.write(f"traffic_bytes_per_launch: {traffic}\n")


def test_traffic_comes_from_the_capture_of_the_exact_variant(tmp_path, monkeypatch):
    prof = tmp_path / "profiles"
    prof.mkdir()
    _summary(prof / "k_element_tma_curved_lake_512_N4.md", "k_element_tma<5,3,2>", 1000)
    _summary(prof / "k_element_pair_curved_lake_512_N4.md", "k_element_pair<5,3>", 2000)
    _summary(prof / "k_element_rows_curved_lake_512_N4.md", "k_element_rows<5,16,2,2>", None)
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.profiled_traffic("k_element_tma<5,3,2>") == 1000
    assert bench.profiled_traffic("k_element_pair<5,3>") == 2000
    # another template instance of a captured kernel, or a summary without
    # the traffic line: no number
    assert bench.profiled_traffic("k_element_pair<5,4>") is None
    assert bench.profiled_traffic("k_element_tma<5,2,2>") is None
    assert bench.profiled_traffic("k_element_rows<5,16,2,2>") is None


def test_committed_traffic_lines_parse():
    """Every committed element-kernel summary that carries a traffic line
    names a variant the engine compiles at N = 4."""
    root = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "profiles")
    for fn in sorted(os.listdir(root)):
        if not (fn.startswith("k_element") and fn.endswith("_curved_lake_512_N4.md")):
            continue
        with open(os.path.join(root, fn)) as f:
            text = f.read()
        title = text.splitlines()[0][2:].split(" ")[0]
        if "traffic_bytes_per_launch:" in text:
            assert title in bench.ELEMENT_KERNELS_N4, fn
            assert bench.profiled_traffic(title) > 0


class _FakeSmi:
    """nvidia-smi's CSV lines, as the sampler reads them at exit."""

    def __init__(self, lines):
        self.lines = lines

    def terminate(self):
        pass

    def communicate(self, timeout=None):
        return "\n".join(self.lines), ""


def test_clocks_keep_the_samples_inside_the_timed_window():
    import datetime
    import time
    now = time.time()

    def row(dt, mhz, watts, cap):
        stamp = datetime.datetime.fromtimestamp(now + dt).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
        return f"{stamp}, {mhz}, 1965, {watts}, 0x0, Not Active, Not Active, Not Active, {cap}"

    lines = [row(-0.2, 1965, 300.0, "Not Active"), row(0.01, 1800, 950.0, "Active"),
             row(0.5, 1700, 990.0, "Active")]
    c = bench.Clocks(0)
    c.proc = _FakeSmi(lines)
    c.window = (now, now + 0.03)
    c.__exit__(None, None, None)
    assert c.result["in_window"] == 1 and c.result["samples"] == 1
    assert c.result["sm_mhz"] == 1800.0 and c.result["reasons"] == ["sw_power_cap"]
    # no sample inside a short window: the nearest one, reported as such
    c = bench.Clocks(0)
    c.proc = _FakeSmi(lines)
    c.window = (now + 0.1, now + 0.12)
    c.__exit__(None, None, None)
    assert c.result["in_window"] == 0 and c.result["sm_mhz"] == 1800.0
    # no window: every sample
    c = bench.Clocks(0)
    c.proc = _FakeSmi(lines)
    c.__exit__(None, None, None)
    assert c.result["samples"] == 3 and c.result["sm_mhz"] == 1800.0
