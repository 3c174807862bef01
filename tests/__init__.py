"""Tests of the B200 hot path (CPU: oracle, lowering, ABI; gpu-marked: device parity)."""
