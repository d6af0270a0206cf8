"""cellweave_b200: cellweave's per-step hot path on one B200 (sm_100a)."""
