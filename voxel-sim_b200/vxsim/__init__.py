"""Host-side model of the Voxel-sim elastic solve on B200.

``materials`` and ``scenes`` describe REV lattices as flat arrays in the layout
of the C ABI (include/vxcorot.h); ``native`` binds libvxcorot.so; ``batched``,
``served`` and ``sharding`` drive the pool, the server and a batch spread over
ranks. The reference's ``solver::`` host API is mirrored in C++ by
voxel-sim_b200/host/vxsim_solver.{hpp,cpp} (libvxsolver.so).
"""
