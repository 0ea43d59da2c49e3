"""Test-only stand-in for the third-party ``sphericart`` package (absent here).

Used only to run the reference implementation in this container when the
golden fixtures are generated.  See ``torch.py``.
"""
