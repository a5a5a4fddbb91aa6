"""Test infrastructure: the restated CPU oracle (oracle.py) and the reference's own CPU engine (ref.py)."""
