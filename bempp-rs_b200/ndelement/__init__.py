"""Minimal stand-in for the parts of the ndelement Python package that bempp uses.

bempp-rs's Python binding imports ``ndelement.reference_cell.ReferenceCellType`` and
``ndelement.ciarlet`` (python/bempp/function_space.py:8-9, python/test/*.py).  Only
Lagrange families of degree 0 and 1 on triangles are needed by the dense assembler.
"""
