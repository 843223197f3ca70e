"""The platform's one-time host algorithms (libb200la.so, no GPU needed) against
the reference's own outputs (golden fixtures) and the oracle, bit for bit."""
import numpy as np
import pytest

CASES = [(2, 8), (2, 17), (3, 4), (3, 7)]
TAGS = [("p", 0), ("pk", 0), ("cd", 1)]


def test_kat_unordered_init_structure(b200):
    # test/LinearAlgebra/CPUsimple_CSR_lMatrix.cc:159-200
    r, c = b200.coo_to_csr(3, [1, 2, 0, 0, 1], [2, 1, 0, 1, 1])
    assert r.tolist() == [0, 2, 4, 5] and c.tolist() == [0, 1, 1, 2, 1]
    r, c = b200.coo_to_csr(3, [2, 0, 0, 1], [1, 0, 1, 1])
    assert r.tolist() == [0, 2, 3, 4] and c.tolist() == [0, 1, 1, 1]


def test_kat_add_values(b200, golden):
    # test/LinearAlgebra/CPUsimple_CSR_lMatrix.cc:79-99
    r, c = b200.coo_to_csr(3, [0, 0, 1, 1, 1, 2, 2], [0, 1, 0, 1, 2, 1, 2])
    v = b200.add_values(r, c, np.zeros(7), [0, 1, 2], [0, 1, 2], np.arange(1.0, 10.0))
    assert v.tolist() == [1, 2, 4, 5, 6, 8, 9]
    assert np.array_equal(v, golden["kat_addvalues_val"])


def test_coo_to_csr_with_values_and_duplicates(b200, oracle):
    rng = np.random.default_rng(3)
    n, nnz = 40, 400
    r = rng.integers(0, n, nnz)
    c = rng.integers(0, n, nnz)   # duplicates included: placement must follow the reference
    v = rng.standard_normal(nnz)
    got = b200.coo_to_csr(n, r, c, v)
    want = oracle.coo_to_csr(n, r, c, v)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)


def test_coo_to_csr_rejects_bad_row(b200):
    with pytest.raises(b200.B200Error) as e:
        b200.coo_to_csr(3, [0, 5], [0, 1])
    assert e.value.code == 5


@pytest.mark.parametrize("dim,N", CASES)
@pytest.mark.parametrize("tag,kind", TAGS)
def test_setup_bit_exact_vs_reference(b200, golden, dim, N, tag, kind):
    key = f"{dim}d{N}_{tag}"
    kc = golden.get(key + "_kcell")
    row, col, val = b200.q1_assemble(dim, N, kind, kc, nu=1e-3, beta=(1.0, 0.5, 0.25))
    assert np.array_equal(row, golden[key + "_row"])
    assert np.array_equal(col, golden[key + "_col"])
    assert np.array_equal(val, golden[key + "_val"])
    nc, sizes, perm = b200.multicoloring(row, col)
    assert np.array_equal(sizes, golden[key + "_mc_sizes"]) and np.array_equal(perm, golden[key + "_mc_perm"])
    nl, lsz, lperm = b200.levelscheduling(row, col)
    assert np.array_equal(lsz, golden[key + "_ls_sizes"]) and np.array_equal(lperm, golden[key + "_ls_perm"])
    ro = b200.reorder_csr(row, col, val, perm)
    for a, s in zip(ro, ("row", "col", "val")):
        assert np.array_equal(a, golden[f"{key}_re_{s}"])
    assert np.array_equal(b200.ilu0(row, col, val), golden[key + "_ilu0"])


def test_rhs_matches_oracle(b200, oracle, golden):
    for dim, N in [(2, 32), (3, 12), (2, 256)]:
        assert np.array_equal(b200.q1_rhs(42, dim, N), oracle.q1_rhs(42, dim, N))
    assert np.array_equal(b200.q1_rhs(42, 2, 32), golden["solve2d32_b"])


@pytest.mark.parametrize("dim,N,kind", [(2, 256, 0), (2, 512, 1), (3, 48, 0)])
def test_full_size_assembly_and_analysis_vs_oracle(b200, oracle, dim, N, kind):
    """Workload-sized systems: assembly, colours and levels equal the oracle's."""
    rng = np.random.default_rng(N)
    kc = np.exp(rng.standard_normal(N ** dim)) if kind == 0 else None
    A = b200.q1_assemble(dim, N, kind, kc, nu=1e-3, beta=(1.0, 0.5))
    B = oracle.q1_assemble(dim, N, kind, kc, nu=1e-3, beta=(1.0, 0.5))
    for a, b in zip(A, B):
        assert np.array_equal(a, b)
    row, col, _ = A
    c1, c2 = b200.multicoloring(row, col), oracle.multicoloring(row, col)
    assert c1[0] == c2[0] and np.array_equal(c1[1], c2[1]) and np.array_equal(c1[2], c2[2])
    if dim == 3:
        assert c1[0] == 8
    l1, l2 = b200.levelscheduling(row, col), oracle.levelscheduling(row, col)
    assert l1[0] == l2[0] and np.array_equal(l1[2], l2[2])


def test_config_structure_bitexact_vs_reference_full_size(b200):
    """The benchmark configurations at their full sizes: the platform's host
    assembly, colouring (3-D 128^3) and level scheduling (2-D 512^2
    convection-diffusion) equal the reference's own (SHA-256 of the arrays
    written by tests/golden/gen_config_counts.py from oracle/_ref)."""
    import hashlib
    import json
    import os

    def sha(*arrays):
        h = hashlib.sha256()
        for a in arrays:
            h.update(np.ascontiguousarray(a).tobytes())
        return h.hexdigest()

    with open(os.path.join(os.path.dirname(__file__), "golden", "config_counts.json")) as f:
        cc = json.load(f)
    row, col, val = b200.q1_assemble(2, 256)
    assert sha(row, col, val) == cc["c1"]["csr_sha256"]
    row, col, val = b200.q1_assemble(3, 128)
    assert sha(row, col, val) == cc["c2"]["csr_sha256"]
    nc, sizes, perm = b200.multicoloring(row, col)
    assert nc == cc["c2"]["colours"] == 8
    assert [int(v) for v in sizes[:nc]] == cc["c2"]["colour_sizes"]
    assert sha(np.asarray(perm, np.int32)) == cc["c2"]["multicoloring_perm_sha256"]
    row, col, val = b200.q1_assemble(2, 512, 1, None, nu=1e-3, beta=(1.0, 0.5))
    assert sha(row, col, val) == cc["c4"]["csr_sha256"]
    nl, lsizes, lperm = b200.levelscheduling(row, col)
    assert nl == cc["c4"]["levels"] == 1537
    assert sha(np.asarray(lsizes[:nl], np.int32)) == cc["c4"]["level_sizes_sha256"]
    assert sha(np.asarray(lperm, np.int32)) == cc["c4"]["levelscheduling_perm_sha256"]
