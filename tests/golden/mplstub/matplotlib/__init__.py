"""Stand-in for matplotlib, used only while generating golden fixtures.

The reference imports ``matplotlib`` (``use("Agg")``) and ``matplotlib.path`` at
module load; neither is installed here and none of the fixture cases draws or
voxelises a polygon, so a no-op ``use`` and a raising ``Path`` suffice.
"""


def use(*args, **kwargs):
    pass
