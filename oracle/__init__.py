"""CPU oracle for the Green-operator matvec and the Fourier-kernel build.

TEST INFRASTRUCTURE ONLY.  This package restates, on the CPU and in FP64, the
algorithms of GilaElectromagnetics.jl (v1.0.3) that the CUDA library replaces.
Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it, and only as the
checker or the timed CPU reference -- never as the thing that is shipped or
measured on the GPU.  The product path (``gilaelectromagnetics.jl_b200``)
never imports this package.

Modules
-------
gla_mem   GlaVol / GlaExtInf / GlaKerOpt restatement   (src/glaMem.jl)
matvec    egoOpr! host path, the 8-branch recursion     (src/glaAct.jl:33-183,
          src/glaActSup.jl:1-1009)
fur       circulant -> egoFur branch extraction, full-spectrum expansion,
          pad-FFT and direct-convolution cross checks   (src/glaMemSup.jl:16-291,
          utl/glaEgoMat.jl:15-77)
synth     seeded synthetic Toeplitz blocks with the Green-function symmetries
kerbuild  ctypes binding of the C restatement of the real-space kernel build
          (src/glaGen.jl, src/glaInt.jl, src/glaIntSup.jl) in ``gen.c``

Parity status: the reference is Julia and cannot run in this container or on
the GPU box (no Julia toolchain).  The matvec restatement is pinned by the
reference's own relational tests (test/extSlfTest.jl: external operator ==
sub-block of the merged self operator; test/oprTest.jl: API contract) and by
agreement (<=1e-13) of three independent formulations: the 8-branch recursion,
the zero-padded FFT convolution and the direct real-space convolution.  No
golden vectors exist in the reference, so absolute parity with the Julia code
is *unpinned* beyond these checks.
"""
