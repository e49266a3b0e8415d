"""B200-native implementation of ABCMB's perturbation + line-of-sight hot path."""
