"""The nvidia_gpu target for the reference's own sources (build_dropin.py; the files under src/)."""
