"""The shared-memory rings of the z-streamed 3D kernel, checked on the CPU by
replaying their index arithmetic (the expressions of stream_kernel in
csrc/ots_stream.cuh) over every depth T, many segment lengths and several
consecutive segments of one CTA.

State ring: NST = 4 stages, copies issued LA = 2 planes ahead; iteration r
(plane k, running index g) reads stage g and, for level 1's y neighbours,
stage g - 1.  Aux ring (Poisson's f): NF = T + 2 slots; f of plane k + 1 is
issued at iteration r, f of plane k - 1 is waited for at the top of r, and
level t reads f of plane k - t.

The packed kernel (stream3p_kernel in csrc/ots_stream3p.cuh) uses the same
two rings with NST = 8 or 4 state stages (copies LA = NST - 2 planes ahead)
and one segment per CTA; it is replayed with those depths below.

Asserted: every read the output depends on finds its plane, already waited
for, in its slot; no copy is issued into a slot that is read in the same
iteration (the copy is asynchronous and may land at once); a copy is only
issued into a slot whose previous plane was waited for (each mbarrier phase
completes before it is re-armed); and every issued copy is waited for by the
end of its segment, or drained on the failure path.
"""
import pytest

NST, LA = 4, 2


def run_segments(T, nits, NST=NST, LA=LA):
    NF = T + 2
    slot = [None] * NF            # plane index (running g) whose copy was issued into the slot
    waited = [True] * NF          # the slot's last issued copy has been waited for
    stage = [None] * NST
    stage_waited = [True] * NST
    rg = 0
    for nit in nits:
        # prologue: state copies for the first LA planes, f of plane kb
        for j in range(min(LA, nit)):
            s = (rg + j) & (NST - 1)
            assert stage_waited[s], "state stage re-armed before its previous phase was waited"
            stage[s], stage_waited[s] = rg + j, False
        if nit > 1:
            s = rg % NF
            assert waited[s], "aux slot re-armed before its previous phase was waited"
            slot[s], waited[s] = rg, False
        for r in range(nit):
            g = rg + r
            # top of the iteration: bounded waits, then the plane barrier
            st = g & (NST - 1)
            assert stage[st] == g
            stage_waited[st] = True
            if r >= 1:
                s = (g - 1) % NF
                assert slot[s] == g - 1, "waiting for an aux plane that was not issued"
                waited[s] = True
            # reads of this iteration (all after the barrier)
            reads_state = {st: g}
            if r >= 1:
                reads_state[(g - 1) & (NST - 1)] = g - 1  # level 1's centre plane
            reads_aux = {}
            for t in range(1, T + 1):
                if r >= 2 * t:  # level t's plane k - t feeds a stored output
                    reads_aux[(g - t) % NF] = g - t
            # copies issued in this iteration
            if r + LA < nit:
                s2 = (g + LA) & (NST - 1)
                assert s2 not in reads_state, "state copy lands in a stage read this iteration"
                assert stage_waited[s2]
                stage[s2], stage_waited[s2] = g + LA, False
            if r + 2 < nit:
                fs = (g + 1) % NF
                assert fs not in reads_aux, "aux copy lands in a slot read this iteration"
                assert waited[fs], "aux slot re-armed before its previous phase was waited"
                slot[fs], waited[fs] = g + 1, False
            for s, plane in reads_state.items():
                assert stage[s] == plane and stage_waited[s]
            for s, plane in reads_aux.items():
                assert slot[s] == plane, "aux slot overwritten before its last needed read"
                assert waited[s], "aux plane read before its copy was waited for"
        # end of segment: nothing left in flight
        assert all(stage_waited), "a state copy of the segment was never waited for"
        assert all(waited), "an aux copy of the segment was never waited for"
        rg += nit


@pytest.mark.parametrize("T", range(1, 9))
def test_stream_rings_never_overwrite_a_live_plane(T):
    for z in (1, 2, 3, 5, 8, 17, 40, 74, 128):
        nit = z + 2 * T  # planes of a segment: its z range plus T of fill each side
        run_segments(T, [nit])
        run_segments(T, [nit, nit, nit - 1 if nit > 2 else nit])


@pytest.mark.parametrize("T", range(1, 5))
@pytest.mark.parametrize("nst", [4, 8])
def test_packed_kernel_rings_never_overwrite_a_live_plane(T, nst):
    # one segment per CTA (the packed kernel's grid covers the z segments)
    for z in (1, 2, 3, 5, 8, 17, 40, 64, 128, 512):
        run_segments(T, [z + 2 * T], NST=nst, LA=nst - 2)


def drain_planes(rg, nit, fail_r, NF):
    """The aux copies the failure path drains (the kernel's loop)."""
    return [j for j in range(fail_r - 1, fail_r + 1) if j < rg + nit - 1 and j >= rg]


@pytest.mark.parametrize("T", [1, 3, 8])
def test_failure_drain_covers_exactly_the_unwaited_aux_copies(T):
    """If the bounded wait at the top of iteration r gives up, the copies
    issued but not yet waited for are f of planes g - 1 (if r >= 1) and g (if
    it was issued, at r - 1); the drain loop visits exactly those."""
    NF = T + 2
    for nit in (2, 3, 7, 20):
        for rg in (0, 11):
            for r in range(nit):
                g = rg + r
                issued = {rg} if nit > 1 else set()
                issued |= {rg + q + 1 for q in range(r) if q + 2 < nit}
                waited = {rg + q - 1 for q in range(1, r)}
                pending = sorted(issued - waited)
                assert drain_planes(rg, nit, g, NF) == pending
