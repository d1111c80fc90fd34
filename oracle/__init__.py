"""CPU oracle for the flexmm 2D FMM evaluation path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / reference leg of ``bench.py`` import anything here, and only
as the checker.  The product package ``flexmm_b200`` never imports it.

* ``oracle.tree``      numpy restatement of flexmm/tree.py
* ``oracle.kifmm``     numpy restatement of flexmm/flexmm2d/{kifmm,fmm,helpers}.py
* ``oracle.kernels``   numpy twins of the reference's example kernels
* ``oracle.direct``    FP64 direct summation in C (OpenMP)
* ``oracle.refimport`` loader for a shimmed copy of the reference itself

The restatement is pinned against outputs of the reference run in the build
container (``tests/golden``, generated by ``tests/golden/make_golden.py``).
"""
