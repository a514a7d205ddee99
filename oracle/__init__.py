"""CPU oracle for the ERK4(3)-IP UPPE/GNLSE propagator.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import this
package, and only as the checker or the timed CPU baseline.  The product
(``project_b200``) never imports it and has no CPU fallback.

Contents (each function cites the reference file:line it restates):

* ``uppe1d``  -- restatement of ``src/1D-ERK4(3)IP UPPE gas/erk43ip_method.py``
  (class ``ERK43IP_UPPE``) with the argon patch of ``gas.py:14-44``.
* ``uppe3d``  -- restatement of ``src/3+1D-UPPE-ERK4(3)IP-envelope/solver_3d.py``
  (class ``ERK43IP_UPPE_3D_Optimized``) and ``media_physics.py`` (``OpticalMedium``,
  ``Argon`` and the CUDA plasma kernel ``media_physics.py:11-67``).
* ``adk``     -- ADK ionisation rate of ``src/THz/2+1D-all field UPPE Argon.py:53-81``.
* ``inputs``  -- seeded synthetic inputs (noise, speckle) that the reference does
  not have; their formulas are defined here and fed identically to the oracle
  and the device.

Parity pinning: ``tests/golden/make_golden.py`` runs the reference's own code
(imported from the reference tree, the 3D solver through a numpy-backed stand-in
for ``cupy`` whose ``RawKernel`` compiles the reference's plasma kernel source
with gcc) on small seeded cases and commits the outputs as fixtures;
``tests/test_oracle_golden.py`` checks this oracle against them.  The features
marked "N-new" (Taylor dispersion medium, ADK LUT in place of the reference's
Keldysh LUT, 1D plasma term, noise, speckle) have no counterpart in the
reference: for them parity is unpinned by any reference test.
"""
