"""CPU model of the device ran1 generator's batch logic (csrc/ran1.cu) against the oracle.

The device produces 32 deviates per warp step: lane l jumps the Park-Miller state by l+1
steps with a modular product, the shuffle table is walked sequentially, and a batch ends
after a step that leaves idum == 0 or iy == 0 (the reference then re-initialises).  This
model follows the kernel lane by lane so the logic is checked without a GPU.
"""

import numpy as np
import pytest

from epsr_python_translation_b200.box import Ran1State
from oracle import oracle

IM = 2147483647


def lcg(d):
    k = d // 127773
    d = 16807 * (d - k * 127773) - 2836 * k
    return d + IM if d < 0 else d


def model(state, n):
    idum, iy, mcall = int(state.idum), int(state.iy), int(state.mcall)
    iv = [int(v) for v in state.iv]
    mul = [pow(16807, lane + 1, IM) for lane in range(32)]
    out = []
    done = 0
    while done < n:
        if idum <= 0 or iy == 0:
            w = (-idum) & 0xFFFFFFFF
            w = w - (1 << 32) if w >= (1 << 31) else w
            d = max(w, 1)
            for j in range(40, 0, -1):
                d = lcg(d)
                if j <= 32:
                    iv[j - 1] = d
            idum, iy = d, iv[0]
        cnt = min(32, n - done)
        idl = [(mul[lane] * idum) % IM for lane in range(32)]
        zeros = [lane for lane in range(cnt) if idl[lane] == 0]
        if zeros:
            cnt = zeros[0] + 1
        s = 0
        while s < cnt:
            j = iy >> 26
            nxt = iv[j]
            iv[j] = idl[s]
            iy = nxt
            out.append(iy)
            s += 1
            if iy == 0:
                break
        cnt = s
        idum = idl[cnt - 1]
        done += cnt
    am = np.float32(4.656612873077393e-10)
    vals = np.array([min(am * np.float32(v), np.float32(0.9999998807907104)) for v in out], np.float32)
    return vals, Ran1State(idum, iy, (mcall + n) & 0xFFFFFFFF, np.array(iv, np.int32))


@pytest.mark.parametrize("seed", [0, -1, -12345, -2147483647, 123, -987654321])
@pytest.mark.parametrize("n", [1, 31, 33, 200])
def test_batched_generator_model_matches_oracle(seed, n):
    st = Ran1State(idum=seed)
    a, sa = model(st, n)
    b, sb = oracle.ran1_fill(st, n)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert sa.idum == sb.idum and sa.iy == sb.iy and np.array_equal(sa.iv, sb.iv)
