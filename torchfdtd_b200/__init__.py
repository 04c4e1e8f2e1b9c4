"""B200-native FDTD engine for TorchFDTD's fused-CUDA path.

Keeps TorchFDTD's ``Project`` / ``Region`` / ``Simulation(project).run()``
API and the ``Region(backend="cuda", cuda_kernel="fused")`` selector. The
time loop runs in hand-written sm_100a CUDA kernels reached through the
C-ABI library ``libtfdtd.so`` (``include/tfdtd.h``); there is no CPU path.
"""
from .models import (Boundaries, BoundaryFace, FieldMonitor, LorentzPole, Material, MeshRefinement, Monitor, Project,
                     Region, RunControl, Source, SourceTimeSettings, SpectrumSettings, Structure, TimeSignal)

__all__ = ['Project', 'Region', 'MeshRefinement', 'Structure', 'Source', 'SourceTimeSettings', 'TimeSignal', 'Monitor',
           'FieldMonitor', 'Material', 'BoundaryFace', 'Boundaries', 'SpectrumSettings', 'LorentzPole', 'RunControl',
           'Simulation', 'Result']


def __getattr__(name):
    # The run API loads the native library on first use, not at import.
    if name in ('Simulation', 'Result'):
        from . import simulation
        return getattr(simulation, name)
    raise AttributeError(name)
