"""Minimal stand-in for the parts of the ndgrid Python package that bempp uses: a
flat-triangle surface grid (points, cells) and the test shapes."""
