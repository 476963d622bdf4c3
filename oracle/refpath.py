"""Where the reference checkout lives (test and build infrastructure only).

One setting for every script that reads the reference's sources or data: the ISSL_REFERENCE
environment variable, defaulting to the read-only checkout of this workspace. The GPU host has no
checkout; nothing that runs there reads it.
"""
import os

REFERENCE = os.environ.get("ISSL_REFERENCE", "/root/reference")
