"""Test infrastructure (oracle): CPU checkers for the CUDA engine; see oracle.py."""
