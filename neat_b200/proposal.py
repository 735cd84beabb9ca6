"""Learned sample proposal (no counterpart in the reference, whose sampler is
uniform stratified: src/structure/HyperTree.cu:347-358).

A tiny MLP (16 -> 32 -> 32 -> 8, SiLU) maps a ray-node segment to the sample
density over 8 equal sub-intervals of [tmin, tmax]; the fused step inverts its
CDF to place a reduced sample budget, and trains it online on the binned
contributions of its uniformly sampled steps (neat_b200/csrc/neat_proposal.cu).
A linear count head on the last hidden layer and the inputs predicts how
much the density varies along the segment (log of its length times the total
variation of its samples' densities); with a count tolerance set, the step
gives flat and empty segments fewer samples than the budget.
Parameters are packed W1 [32][16] | b1 [32] | W2 [32][32] | b2 [32] |
W3 [8][32] | b3 [8] | Wv [32] | Uv [16] | bv.
"""
import torch

from . import _lib


def proposal_init(generator=None):
    """kaiming_normal (fan_in) hidden weights, zero biases, and a zero output
    layer, so that the untrained proposal is uniform; a zero count head
    (v = 0: every segment keeps the budget's count until it is trained)."""
    H, I, B = _lib.NEAT_PROPOSAL_HIDDEN, _lib.NEAT_PROPOSAL_IN, _lib.NEAT_PROPOSAL_BINS
    w1 = torch.randn((H, I), generator=generator) * (2.0 / I) ** 0.5
    w2 = torch.randn((H, H), generator=generator) * (2.0 / H) ** 0.5
    return torch.cat([w1.reshape(-1), torch.zeros(H), w2.reshape(-1), torch.zeros(H), torch.zeros(B * H),
                      torch.zeros(B), torch.zeros(H + I + 1)]).to(torch.float32)
