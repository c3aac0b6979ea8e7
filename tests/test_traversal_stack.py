"""The warp-cooperative traversal's stack bound (smallupbp_b200/csrc/upbp_traverse.cuh).

A model of the pop policy of `warp_traverse`, run on the worst case for the stack: a full binary
tree of the largest depth an LBVH over 62-bit keys can have, every box hit.  Each step pops `take`
nodes from the top of the stack and pushes both children of each; with the bounded `take` the
stack never exceeds its 1024 entries, while popping 32 at a time regardless overflows it.
"""
STACK, MAX_DEPTH, WARP = 1024, 64, 32
LEAF_LEVEL = 62  # internal nodes along a root-to-leaf path: split prefix lengths 2..63


def max_stack(bounded: bool, steps: int = 200_000) -> int:
    stack, top = [0], 1  # depths of the pending internal nodes
    for _ in range(steps):
        if not stack:
            break
        sp = len(stack)
        take = min(sp, WARP)
        if bounded:
            take = min(take, max(1, STACK - MAX_DEPTH - sp))
        popped = stack[sp - take:]
        del stack[sp - take:]
        for d in popped:
            if d + 1 < LEAF_LEVEL:
                stack += [d + 1, d + 1]
        top = max(top, len(stack))
    return top


def test_bounded_pop_never_overflows():
    assert max_stack(True) <= STACK


def test_unbounded_pop_would_overflow():
    assert max_stack(False, steps=5_000) > STACK
