"""Merging independent problems into one block-diagonal problem (CPU)."""

from __future__ import annotations

import torch

import torchls_b200 as tls
from torchls_b200 import synthetic
from torchls_b200.batched import merge_problems


def test_merge_offsets_and_data():
    datas = synthetic.batched_bundle_adjustment(4, first_seed=3)
    probs = [synthetic.build_bundle_adjustment(d, tls, loss=tls.HuberLoss(0.01)) for d in datas]
    merged, var_problem, slices = merge_problems(probs)
    for name in ("cams", "points"):
        assert merged.parameters[name].shape[0] == sum(p.parameters[name].shape[0] for p in probs)
        assert torch.equal(torch.bincount(var_problem[name]),
                           torch.tensor([p.parameters[name].shape[0] for p in probs]))
    for j, p in enumerate(probs):
        for name in ("cams", "points"):
            assert torch.equal(merged.parameters[name][slices[j][name]], p.parameters[name])
    for k in range(len(probs[0]._costs)):
        n = sum(int(torch.as_tensor(p._costs[k].args[1].id).numel()) for p in probs)
        ids = torch.as_tensor(merged._costs[k].args[1].id)
        assert ids.numel() == n
        # point indices point into each problem's own block of the merged group
        start = 0
        for j, p in enumerate(probs):
            m = int(torch.as_tensor(p._costs[k].args[1].id).numel())
            block = ids[start : start + m]
            assert int(block.min()) >= slices[j]["points"].start and int(block.max()) < slices[j]["points"].stop
            start += m
