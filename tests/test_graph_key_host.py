"""A captured cross-body batch (CUDA graph) holds every device address it was
captured with, so its key must cover every buffer the captured sequence
touches: a buffer that moves (grows) must change the key, or a later replay
would read and write freed memory. Checked on the sources: every device
pointer of the mixed-precision workspace (MixedWork, TcWork) and every
context buffer of a ragged batch appears in the key (nemoh_b200/csrc/api.cu,
the `sig` vector of ragged_batch)."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "nemoh_b200", "csrc")


def _read(name):
    with open(os.path.join(CSRC, name)) as f:
        return f.read()


def _struct_pointers(src, name):
    body = src[src.index("struct %s {" % name):]
    body = body[:body.index("\n};")]
    return re.findall(r"^\s*(?:[\w:]+\s+)*[\w:]+\s*\*\s*(\w+)\s*=\s*nullptr;", body, re.M)


def _key_block():
    api = _read("api.cu")
    start = api.index("std::vector<long long> sig = {")
    return api[start:api.index("};", start)]


def test_mixed_workspace_buffers_are_in_the_graph_key():
    key = _key_block()
    mixed = _struct_pointers(_read("mixed.cuh"), "MixedWork")
    tc = _struct_pointers(_read("tc_gemm.cuh"), "TcWork")
    assert {"lu", "norms", "flow", "act"} <= set(mixed) and {"a", "b", "wv"} <= set(tc)
    # status points at the context's status word, allocated once with the context
    missing = [f for f in mixed if f != "status" and "c->mixed.%s" % f not in key]
    missing += [f for f in tc if "c->mixed.tc.%s" % f not in key]
    assert not missing, missing


def test_context_buffers_of_a_ragged_batch_are_in_the_graph_key():
    key = _key_block()
    for buf in ("d_D", "d_S", "d_X", "d_Y", "d_diag", "d_inv", "d_oms", "d_slots", "d_smesh", "d_items",
                "d_roff", "d_rord", "d_flow"):
        assert "c->%s.p" % buf in key, buf
