"""Learned value surrogate (BF16 MLP) trained and queried with libpe_b200."""
