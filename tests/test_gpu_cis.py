"""Per-(gene, variant) cis genotype statistics (gpl_cis_stats) against the per-cell score statistics
(gpl_score_stats, checked against the reference's getScoreStats on the golden cases): for every
gene, its own variants' donor dosages expanded to the cells give the same statistic through both
paths (group sums of donor-constant columns versus per-cell sums), within 1e-8 relative; the
likelihood ratio is the statistic's square; and the causal variants of the synthetic genes with
a genotype effect score above the null ones."""
import numpy as np
import pytest

from gaspacho2_b200 import GPLVM, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fitted():
    # 6,000 cells over 4 batches x 300 donors: at most 1,200 batch x donor cell groups, few enough
    # (<= N/4 + 1) for the categorical variables to be handled by group sums
    return synth.make(4, 1, N=6000, G=24, M=8, Q=2, init=True)


def test_cis_statistics_equal_per_cell_scores(fitted):
    ds = fitted
    donor_var = len(ds.z.c) - 1  # the donor is the design's last variable
    donor = ds.z.columns[donor_var]
    D, J, V = ds.genotypes.shape
    with GPLVM.from_dataset(ds) as m:
        m.set_params(ds.init)
        m.kernel_mats()
        m.glm_init()
        m.irls(0, 30)
        S, LR = m.cis_stats(ds.genotypes, donor_var)
        assert np.all(np.isfinite(S))
        assert np.allclose(LR, S * S, rtol=1e-14, atol=0)
        worst = 0.0
        for j in range(J):
            Gc = ds.genotypes[donor, j, :].astype(np.float64)  # N x V: the cells' dosages of gene j's variants
            Sj = m.score_stats(Gc)[j]
            e = np.max(np.abs(S[j] - Sj) / np.maximum(np.abs(Sj), 1.0))
            worst = max(worst, e)
        print(f"worst difference against the per-cell statistics: {worst:.2e}")
        assert worst <= 1e-8


def test_causal_variants_stand_out():
    ds = synth.make(4, 2, N=6000, G=60, M=8, Q=2, init=True)
    donor_var = len(ds.z.c) - 1
    truth = ds.geno_truth
    with GPLVM.from_dataset(ds) as m:
        m.set_params(ds.init)
        m.kernel_mats()
        m.glm_init()
        m.irls(0, 40)
        _, LR = m.cis_stats(ds.genotypes, donor_var)
    J, V = LR.shape
    strong = np.abs(truth["main"]) > 0.12
    causal_lr = LR[np.arange(J), truth["causal"]]
    mask = np.ones_like(LR, bool)
    mask[np.arange(J), truth["causal"]] = False
    print(f"median LR: causal variants of strong-effect genes {np.median(causal_lr[strong]):.2f}, "
          f"non-causal variants {np.median(LR[mask]):.2f}")
    assert np.median(causal_lr[strong]) > 3.0 * np.median(LR[mask])
