"""Host-side model of the Voxel-sim elastic solve on B200.

``materials`` and ``scenes`` describe REV lattices as flat arrays in the layout
of the C ABI (include/vxcorot.h); ``native`` binds libvxcorot.so; ``solver``
mirrors the reference's ``solver::`` host API over it.
"""
