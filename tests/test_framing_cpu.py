"""Payload framing rules that need no GPU: how many stripes a payload fills, the tape
outer coder's shape k = ceil(groups / 3), m = groups - k, and its shard size
ceil(segment / k) rounded up to 64 with the 4 MiB ceiling
(benches/gf16-bench/src/bin/live.rs:1-16)."""
import pytest


def test_frame_stripe_count(rsb):
    assert rsb.frame_stripe_count(0, 32, 987) == 0
    assert rsb.frame_stripe_count(1, 32, 987) == 1
    assert rsb.frame_stripe_count(32 * 987, 32, 987) == 1
    assert rsb.frame_stripe_count(32 * 987 + 1, 32, 987) == 2
    assert rsb.frame_stripe_count(10 ** 6, 32, 987) == 32
    assert rsb.frame_stripe_count(100, 0, 987) == 0
    assert rsb.frame_stripe_count(100, 4, 0) == 0


@pytest.mark.parametrize("groups,k,m", [(2, 1, 1), (3, 1, 2), (4, 2, 2), (20, 7, 13), (21, 7, 14),
                                        (300, 100, 200), (65536, 21846, 43690)])
def test_outer_shape(rsb, groups, k, m):
    assert rsb.outer_shape(groups) == (k, m)


@pytest.mark.parametrize("groups,err", [(0, "TooFewDataShards"), (1, "TooFewParityShards"),
                                        (65537, "TooManyShards")])
def test_outer_shape_errors(rsb, groups, err):
    with pytest.raises(rsb.RsError) as e:
        rsb.outer_shape(groups)
    assert e.value.name == err


def test_outer_shard_bytes(rsb):
    assert rsb.outer_shard_bytes(0, 7) == 64
    assert rsb.outer_shard_bytes(1, 7) == 64
    assert rsb.outer_shard_bytes(7 * 64, 7) == 64
    assert rsb.outer_shard_bytes(7 * 64 + 1, 7) == 128
    assert rsb.outer_shard_bytes(10 ** 6, 7) == 142912  # ceil(1e6 / 7) = 142858 -> 142912
    assert rsb.outer_shard_bytes(7 * (4 << 20), 7) == 4 << 20
    with pytest.raises(rsb.RsError) as e:
        rsb.outer_shard_bytes(7 * (4 << 20) + 1, 7)
    assert e.value.name == "TooLarge"
    with pytest.raises(rsb.RsError) as e:
        rsb.outer_shard_bytes(100, 0)
    assert e.value.name == "TooFewDataShards"
