"""Compact eight-state semi-Lagrangian contact game on the GPU
(the local pair game of src/pursuit_evasion/local_game)."""
