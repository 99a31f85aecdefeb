"""Seeded synthetic workloads in the shapes the scan is benchmarked on.

The real plant-genome data these shapes stand for is not available, so every
reference and sample is generated from a seed (see include/ibs_tools.h):

* plain_1mbp   -- 1 Mbp reference in 2 contigs, i.i.d. ACGT, 0.1% N in runs
                  of 50-500 bp; one sample = canonical k=25 k-mers of a copy
                  with 1% i.i.d. SNPs plus 5% random k-mers (~1.05M), counts
                  2-255, KMC p=5 / 512 bins; window 50 kbp. CPU-runnable.
* plain_2gbp   -- 2 Gbp reference in 10 contigs of 100-400 Mbp, 0.5% N runs;
                  one sample of ~2e9 k=25 k-mers from a copy cut into 1 Mbp
                  blocks whose SNP rate is 0.01/0.5/2/5% with probability
                  0.2/0.4/0.3/0.1, plus 10% random k-mers; KMC p=9 (4-byte
                  suffix records) / 512 bins; window 50 kbp.
* panel_4gbp   -- 4.2 Gbp reference in 7 contigs of 450-750 Mbp, 1% N runs;
                  16 samples of 0.3e9-2.1e9 k=31 k-mers (log-uniform sizes via
                  block presence), own seeds, 2-5 introgression blocks of
                  1-20 Mbp at 0.01%; KMC p=7.
* served_2gbp  -- the plain_2gbp reference and 16 samples of its block model
                  with their own seeds, log-uniform 0.15e9-1.0e9 k=25 k-mers:
                  the served stream's resident pool.
* admitted_4gbp -- the panel_4gbp reference and 48 samples of 0.5e9-2.1e9
                  k=31 k-mers (optionally scaled): the memory-admitted pool,
                  several times the memory the server may use.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import RefSpec, SampleSpec

MB = 1_000_000


@dataclass
class Workload:
    name: str
    ref: RefSpec
    samples: list
    kmc: dict
    window: int = 50_000
    description: str = ""
    extra: dict = field(default_factory=dict)

    @property
    def k(self) -> int:
        return self.samples[0].k


BLOCK_RATES = (0.0001, 0.005, 0.02, 0.05)
BLOCK_PROBS = (0.2, 0.4, 0.3, 0.1)


def plain_1mbp() -> Workload:
    ref = RefSpec(seed=1, lens=[600_000, 400_000], n_frac=0.001, n_run=(50, 500),
                  names=["chr1", "chr2"])
    smp = SampleSpec(seed=101, k=25, class_rate=(0.01,), class_prob=(1.0,), block_len=1 << 20,
                     random_frac=0.05)
    return Workload("plain_1mbp", ref, [smp], dict(k=25, p=5, sig_len=9, n_bins=512, counter_size=1),
                    description="1 Mbp x ~1.05M k=25 k-mers, W=50 kbp")


PLAIN_2GBP_LENS = [300, 150, 250, 100, 400, 180, 220, 120, 160, 120]


def plain_2gbp(scale: float = 1.0) -> Workload:
    lens = [int(x * MB * scale) for x in PLAIN_2GBP_LENS]
    ref = RefSpec(seed=2, lens=lens, n_frac=0.005, n_run=(50, 500),
                  names=[f"chr{i + 1}" for i in range(len(lens))])
    smp = SampleSpec(seed=202, k=25, class_rate=BLOCK_RATES, class_prob=BLOCK_PROBS,
                     block_len=1 * MB, random_frac=0.10)
    return Workload("plain_2gbp" if scale == 1.0 else f"plain_2gbp_x{scale:g}", ref, [smp],
                    dict(k=25, p=9, sig_len=9, n_bins=512, counter_size=1),
                    description=f"{sum(lens) / 1e9:.3g} Gbp x ~{2.2 * scale:.3g}e9 k=25 k-mers, W=50 kbp")


PANEL_4GBP_LENS = [750, 450, 600, 700, 550, 650, 500]


def panel_4gbp(n_samples: int = 16, scale: float = 1.0, sample_scale: float = 1.0) -> Workload:
    lens = [int(x * MB * scale) for x in PANEL_4GBP_LENS]
    ref = RefSpec(seed=3, lens=lens, n_frac=0.01, n_run=(50, 500),
                  names=[f"chr{i + 1}H" for i in range(len(lens))])
    rng = np.random.default_rng(303)
    positions = sum(lens)
    samples = []
    for s in range(n_samples):
        target = math.exp(rng.uniform(math.log(0.3e9), math.log(2.1e9))) * scale * sample_scale
        present = min(1.0, target / (positions * 1.10))
        intro = []
        for _ in range(int(rng.integers(2, 6))):
            c = int(rng.integers(0, len(lens)))
            ln = int(rng.integers(1 * MB, 20 * MB) * scale)
            st = int(rng.integers(0, max(1, lens[c] - ln)))
            intro.append((c, st, ln))
        samples.append(SampleSpec(seed=3000 + s, k=31, class_rate=BLOCK_RATES, class_prob=BLOCK_PROBS,
                                  block_len=1 * MB, present_frac=present, random_frac=0.10 * present,
                                  intro=intro, intro_rate=0.0001))
    name = "panel_4gbp" if sample_scale == 1.0 else f"panel_4gbp_samples_x{sample_scale:g}"
    return Workload(name, ref, samples, dict(k=31, p=7, sig_len=9, n_bins=512, counter_size=1),
                    description=f"4.2 Gbp x {n_samples} samples of {0.3 * sample_scale:g}e9-"
                                f"{2.1 * sample_scale:g}e9 k=31 k-mers, W=50 kbp")


def served_2gbp(n_samples: int = 16, scale: float = 1.0) -> Workload:
    """The served stream's pool: the plain_2gbp reference and n samples made
    by its block-divergence model with their own seeds, sized log-uniform
    0.15e9-1.0e9 k=25 k-mers (panel_4gbp's 0.3e9-2.1e9 scaled to the 2 Gbp
    reference), so that all of them stay resident on one GPU."""
    base = plain_2gbp(scale)
    rng = np.random.default_rng(404)
    positions = sum(base.ref.lens)
    samples = []
    for s in range(n_samples):
        target = math.exp(rng.uniform(math.log(0.15e9), math.log(1.0e9))) * scale
        samples.append(SampleSpec(seed=4000 + s, k=25, class_rate=BLOCK_RATES, class_prob=BLOCK_PROBS,
                                  block_len=1 * MB, present_frac=min(1.0, target / (positions * 1.10)),
                                  random_frac=0.10 * min(1.0, target / (positions * 1.10))))
    return Workload("served_2gbp" if scale == 1.0 else f"served_2gbp_x{scale:g}", base.ref, samples,
                    base.kmc, description=f"{sum(base.ref.lens) / 1e9:.3g} Gbp x {n_samples} samples of "
                                          f"0.15e9-1.0e9 k=25 k-mers, W=50 kbp")


def admitted_4gbp(n_samples: int = 48, scale: float = 1.0, sample_scale: float = 1.0) -> Workload:
    """Memory-admitted serving pool: the panel_4gbp reference and n samples of
    0.5e9-2.1e9 k=31 k-mers (log-uniform, times sample_scale), made by the
    block-divergence model with their own seeds; together several times the
    device memory a server is given."""
    base = panel_4gbp(n_samples=1, scale=scale)
    rng = np.random.default_rng(505)
    positions = sum(base.ref.lens)
    samples = []
    for s in range(n_samples):
        target = math.exp(rng.uniform(math.log(0.5e9), math.log(2.1e9))) * scale * sample_scale
        samples.append(SampleSpec(seed=5000 + s, k=31, class_rate=BLOCK_RATES, class_prob=BLOCK_PROBS,
                                  block_len=1 * MB, present_frac=min(1.0, target / (positions * 1.10)),
                                  random_frac=0.10 * min(1.0, target / (positions * 1.10))))
    name = "admitted_4gbp" + ("" if sample_scale == 1.0 else f"_samples_x{sample_scale:g}")
    return Workload(name, base.ref, samples, base.kmc,
                    description=f"4.2 Gbp x {n_samples} samples of {0.5 * sample_scale:g}e9-"
                                f"{2.1 * sample_scale:g}e9 k=31 k-mers, W=50 kbp")
