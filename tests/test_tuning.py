"""The CTA class table the engine compiles in (python_b200/csrc/cta_classes.inc)
is a valid autotuner result: ascending orders, each class one of the timed
candidates, and in agreement with the tuner's record when there is one."""
import json

from python_b200 import autotune


def test_class_table_comes_from_the_candidates():
    classes = autotune.parse_classes()
    cands = set(autotune.parse_candidates())
    orders = [c[0] for c in classes]
    assert orders == sorted(set(orders)) and orders[0] > 32
    assert orders[-1] >= 1024                      # every supported order has a class
    for c in classes:
        assert c in cands, c


def test_record_matches_table():
    if not autotune.RECORD.exists():
        return
    rec = json.loads(autotune.RECORD.read_text())
    table = {c[0]: c for c in autotune.parse_classes()}
    for entry in rec["classes"]:
        assert tuple(entry["chosen"]) == table[entry["P"]], entry["P"]
        timed = [tuple(c["config"]) for c in entry["candidates"] if "ms" in c]
        assert tuple(entry["chosen"]) in timed


def test_candidates_of_one_order_share_storage_and_chunk_width():
    # an inverse fuses its left-of-panel updates per column in shared memory and
    # per CC-wide chunk in the workspace: those two choices fix the bits
    by_p = {}
    for c in autotune.parse_candidates():
        by_p.setdefault(c[0], set()).add((c[5], c[3] if c[5] else None))
    for p, kinds in by_p.items():
        assert len(kinds) == 1, (p, kinds)


def test_certified_class_table_comes_from_the_candidates():
    """Every certified class is one of the tuner's candidate shapes, in order of P."""
    cands = set(autotune.parse_cgj_candidates())
    classes = autotune.parse_cgj_classes()
    assert classes, "no certified classes"
    assert [c[0] for c in classes] == sorted({c[0] for c in classes})
    for c in classes:
        assert c in cands, c


def test_certified_record_matches_table():
    """When the certified classes were tuned, the table is the record's winners
    at the class edges the record kept."""
    if not autotune.RECORD.exists():
        return
    rec = json.loads(autotune.RECORD.read_text()).get("cgj")
    if rec is None:
        return
    chosen = {e["P"]: tuple(e["chosen"]) for e in rec["classes"]}
    dropped = {e["P"] for e in rec["edges"] if e["dropped"]}
    table = autotune.parse_cgj_classes()
    assert sorted(set(chosen) - dropped) == [c[0] for c in table]
    for c in table:
        assert chosen[c[0]] == tuple(c), (chosen[c[0]], c)


def test_small_class_table_comes_from_the_candidates():
    cands = set(autotune.parse_small_candidates())
    classes = autotune.parse_small_classes()
    assert classes and classes[-1][0] == 32, "orders up to 32 stay on the small family"
    assert [c[0] for c in classes] == sorted({c[0] for c in classes})
    for np_, g in classes:
        assert (np_, g) in cands and np_ <= g and g in (4, 8, 16, 32)


def test_small_record_matches_table():
    if not autotune.RECORD.exists():
        return
    rec = json.loads(autotune.RECORD.read_text()).get("small")
    if rec is None:
        return
    chosen = {e["NP"]: tuple(e["chosen"]) for e in rec["classes"]}
    dropped = {e["NP"] for e in rec["edges"] if e["dropped"]}
    table = autotune.parse_small_classes()
    assert sorted(set(chosen) - dropped) == [c[0] for c in table]
    for c in table:
        assert chosen[c[0]] == tuple(c)
