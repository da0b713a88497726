"""lpm_b200 -- B200-native LPM linear solve (matrix-free K.u inside CG/PCG, adjoint gradient, serving loop).

Host layer over the CUDA library ``liblpm_b200.so`` (C ABI, see ``include/lpm_b200.h``).  Modules mirror the
reference's public modules so that callers can switch with a changed import:

    geom         lattice geometry / BCs / material maps   (coarse3d/geom3d.py, coarse2d/lin2d.py, coarse2d/cg.py)
    lin3d        solve_pcg / Lattice3D on the GPU          (coarse3d/lin3d.py)
    lin2d        matrix-free 2D solves; stiffness + solve_disp on an assembled CSR K
                                                           (coarse2d/lin2d.py, timing/t2d/solver2d.py, cg2plain.py)
    torch_lpm3d  SCT, LinSolve, LoadSet, CoarseT, FineRefT (coarse3d/torch_lpm3d.py)
    torch_v1     SCTV, CoarseTV, FineRefTV: per-specimen voids (cement3d/torch_v1.py)
    train3d      Scatter, group_penalty: bond-parameter assembly (coarse3d/train3d.py)
    torch_lpm    2D CoarseT (matrix-free + adjoint)        (coarse2d/torch_lpm.py)
    amg          AMGGeom, AMG3D, AmgBatch                  (timing/t3d/amg3d.py)
    fine_data    data/fine_*.npz generation                (coarse3d/gen_fine.py)
    serve        continuous-batching solve service         (no counterpart)
    micro        seeded synthetic microstructures          (coarse2d/micro.py, coarse3d/micro3d.py)
"""
__version__ = "0.1.0"
