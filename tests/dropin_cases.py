"""Inputs and expectations shared by the drop-in tests: packs as the
reference's load-balanced walk makes them, and particle time-step levels with
the rule deciding which particles an active-level pass changes."""
import numpy as np


def lb_packs(tl, nsub, leaf_base):
    """Packs as the reference's load-balanced walk makes them
    (add_one_p2ppack, src/fmm_LB.c:25-49): the entries whose sink and source
    both lie in one of nsub contiguous leaf ranges (subtrees) form that
    range's pack, the remaining entries one last inter-subtree pack; each
    pack's leaf and particle range spans its smallest to largest leaf id, so
    the inter-subtree pack overlaps the others."""
    L = tl.nleaf
    cut = np.linspace(0, L, nsub + 1).astype(np.int64)
    sub_t = np.searchsorted(cut, tl.task_t, side="right") - 1
    sub_s = np.searchsorted(cut, tl.task_s, side="right") - 1
    groups = [np.nonzero((sub_t == k) & (sub_s == k))[0] for k in range(nsub)]
    groups.append(np.nonzero(sub_t != sub_s)[0])
    packs = []
    for g in groups:
        if g.size == 0:
            continue
        t, s = tl.task_t[g], tl.task_s[g]
        lo, hi = int(min(t.min(), s.min())), int(max(t.max(), s.max()))
        packs.append(dict(task_t=t + leaf_base, task_s=s + leaf_base, ileaf=lo + leaf_base, nleaf=hi - lo + 1,
                          ipart=int(tl.leaf_ipart[lo]),
                          npart=int(tl.leaf_ipart[hi] - tl.leaf_ipart[lo] + tl.leaf_npart[hi])))
    return packs


def act_levels(tl, g):
    """Time-step levels as a hierarchical stepper assigns them: one level
    per leaf for most particles (neighbours share a step), 5% of the
    particles on another level (0-3), 2% on level 255."""
    n = tl.pos.shape[1]
    act = np.zeros(n, np.int32)
    lvl = g.integers(1, 4, tl.nleaf)
    for l in range(tl.nleaf):
        act[tl.leaf_ipart[l]:tl.leaf_ipart[l] + tl.leaf_npart[l]] = lvl[l]
    flip = g.uniform(size=n) < 0.05
    act[flip] = g.integers(0, 4, int(flip.sum()))
    act[g.uniform(size=n) < 0.02] = 255
    return act


def act_updates(act, level, kernel_filter):
    """The particles an active-level pass changes: the reference's download
    adds where level == -1 or (level != 0 and act == level)
    (src/gpu_func.impl.h:644-653); with ACT_OPT its chunked pass's kernel
    leaves a sink at zero unless act and level agree as bytes
    (src/gpu_kernel.impl.h:392-396)."""
    upd = (level == -1) | ((level != 0) & (act == level))
    if kernel_filter:
        upd &= (act & 0xFF) == (level & 0xFF)
    return upd
