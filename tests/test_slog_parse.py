"""The program-description route (CPU): the generator's parser on a synthetic
program written in the reference's generated style (comments, lambdas, SCCs added
out of creation order), the description reader, and the builder on the oracle."""
import os
import sys

import numpy as np
import pytest

import oracle as O
import parallel_ra_b200 as P
from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_slog_golden as G  # noqa: E402

SOURCE = r'''
#include "../src/parallel_RA_inc.h"
int main(int argc, char **argv)
{
relation* rel_e_2_1_2 = new relation(1, true, 2, 256, "rel_e_2_1_2", "../data/toy//e_2_1.dat", FULL);
relation* rel_p_2_1_2 = new relation(1, true, 2, 257, "rel_p_2_1_2", "../data/toy//p_2_2.dat", FULL);
relation* rel_q_2_2_1 = new relation(1, false, 2, 257, "rel_q_2_2_1", "../data/toy//q_2_3.dat", FULL);
RAM* scc2 = new RAM(true, 2);
scc2->add_relation(rel_p_2_1_2, true);
scc2->add_relation(rel_e_2_1_2, false);
scc2->add_rule(new parallel_join(rel_p_2_1_2, rel_p_2_1_2, DELTA, rel_e_2_1_2, FULL, {3, 1}));
// scc2->add_rule(new parallel_copy(rel_p_2_1_2, rel_e_2_1_2, FULL, {0, 1}));
RAM* scc1 = new RAM(false, 1);
scc1->add_relation(rel_p_2_1_2, true);
scc1->add_relation(rel_e_2_1_2, false);
scc1->add_relation(rel_q_2_2_1, true);
scc1->add_rule(new parallel_copy(rel_p_2_1_2, rel_e_2_1_2, FULL, {1, 0}));
scc1->add_rule(new parallel_copy_filter(rel_q_2_2_1, rel_e_2_1_2, FULL, {1, 2}, [](const u64* const data){ return !(data[0] == data[1]); }));
/* scc1->add_rule(new parallel_acopy(rel_q_2_2_1, rel_p_2_1_2, DELTA, {1, 0, 2})); */
LIE* lie = new LIE();
lie->add_scc(scc1);
lie->add_scc(scc2);
lie->add_scc_dependance(scc1, scc2);
lie->set_batch_size(3);
}
'''


def test_parser_reads_generated_style_source():
    lines, rels = G.parse_program(SOURCE)
    assert lines[0] == "batch 3"
    assert [r["name"] for r in rels] == ["rel_e_2_1_2", "rel_p_2_1_2", "rel_q_2_2_1"]
    assert "rel 1 1 2 256 FULL rel_e_2_1_2 e_2_1.dat" in lines
    # SCCs in LIE::add_scc order (scc1 first), commented rules ignored
    assert [l for l in lines if l.startswith("scc")] == ["scc 0 1", "scc 1 2"]
    rules = [l for l in lines if l.startswith(("join", "copy"))]
    assert rules == ["join 1 1 1 DELTA 0 FULL 3,1", "copy 0 copy 1 0 FULL - 1,0", "copy 0 filter 2 0 FULL ne 1,2"]
    assert "dep 0 1" in lines


def _write_toy(tmp_path):
    lines, _ = G.parse_program(SOURCE)
    (tmp_path / "program.txt").write_text("\n".join(lines) + "\n")
    rng = np.random.default_rng(4)
    e = np.concatenate([rng.integers(0, 30, size=(60, 2)), np.arange(60)[:, None]], axis=1).astype(np.uint64)
    P.datagen.write_relation(str(tmp_path / "e_2_1.dat"), e)
    for f in ("p_2_2.dat", "q_2_3.dat"):
        P.datagen.write_empty_relation(str(tmp_path / f))
    return e


def test_described_program_on_the_oracle_is_a_closure(tmp_path):
    """The toy program: p = reversed e, then p's closure over e; q = the edges with
    distinct endpoints, projected (dst, id)."""
    e = _write_toy(tmp_path)
    o = O.OracleProgram()
    h = P.programs.build_described(o, str(tmp_path / "program.txt"), str(tmp_path))
    assert h.pop("__batch__") == 3
    o.execute(3)
    q = o.dump_full(h["rel_q_2_2_1"])
    want_q = {(int(b), int(i)) for a, b, i in e if a != b}
    assert {(int(r[0]), int(r[1])) for r in q} == want_q
    assert [sid for sid, _ in o.history()] == [1, 2]
    o.close()


def test_description_rejects_a_file_of_the_wrong_width(tmp_path):
    _write_toy(tmp_path)
    P.datagen.write_relation(str(tmp_path / "e_2_1.dat"), np.zeros((3, 4), dtype=np.uint64))
    o = O.OracleProgram()
    with pytest.raises(ValueError):
        P.programs.build_described(o, str(tmp_path / "program.txt"), str(tmp_path))
    o.close()
