"""CPU oracle -- test infrastructure only (tests/, smoke(), bench.py's CPU baseline)."""
