"""Test oracle for the distance-driven projector path (test infrastructure:
imported only by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline; never by the product package)."""
