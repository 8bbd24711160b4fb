"""Test infrastructure: the CPU oracle of the reference's IF-RK step (see gbght_oracle.py)."""
