"""bench.py's roofline bookkeeping, on the host: the per-kernel algorithmic bytes add up to the
step's, and every DRAM-traffic / instruction-mix entry of profiles/ncu_traffic.json is matched to
the kernel the bench line names for that stage (same kernel, same pair action), so a capture of
one kernel is never reported for another."""
import importlib.util
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    argv = sys.argv
    sys.argv = ["bench.py"]
    try:
        spec.loader.exec_module(mod)
    finally:
        sys.argv = argv
    return mod


def test_stage_bytes_add_up_to_the_step():
    """2D: 189 B exactly; 3D: the stages add up to 244.5 B, which the step figure quotes rounded
    to 245 B."""
    b = _bench()
    for dim in (2, 3):
        total = sum(v[dim] for v in b.B_ALG_STAGE.values())
        assert abs(total - b.B_ALG_STEP[dim]) <= (0.0 if dim == 2 else 0.5), (dim, total)


def test_kernel_key_of_labels_and_ncu_names():
    b = _bench()
    assert b.kernel_key("k_list<CPMom> (momentum)") == ("k_list", "CPMom")
    assert b.kernel_key("k_list<2, CPMom<2, 1, 0>, 1>") == ("k_list", "CPMom")
    assert b.kernel_key("k_win_build<CPCont<2, 1, 0>>") == ("k_win_build", "CPCont")
    assert b.kernel_key("k_build<3>") == ("k_build", None)
    assert b.kernel_key("k_build (neighbour lists + nCount)") == ("k_build", None)
    assert b.kernel_key("k_list<CPCont> (x)") != b.kernel_key("k_list<CPMom> (x)")


def test_traffic_entries_name_the_kernels_of_their_stage():
    b = _bench()
    with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
        traffic = json.load(f)
    # the default 2D line: window search (continuity inside it) and the list momentum pass
    labels_2d = dict(b.KERNEL_OF_STAGE)
    labels_2d["search"] = "k_win_build<CPCont> (window search)"
    for stage, e in traffic["2d"].items():
        assert b.kernel_key(e["kernel"]) == b.kernel_key(labels_2d[stage]), (stage, e["kernel"])
    for case in ("3d", "3d-small"):
        for stage, e in traffic[case].items():
            assert b.kernel_key(e["kernel"]) == b.kernel_key(b.KERNEL_OF_STAGE[stage]), (case, stage, e["kernel"])
    for case in traffic.values():
        for e in case.values():
            assert e["bytes_per_launch"] > 0 and e["warp_inst_per_launch"] > 0 and e["flops_per_launch"] > 0
