"""CPU oracle: a numpy restatement of DeePAW-HALF's fixed-density PAW path.

TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library imports, links or
executes this package; only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` use it, and there
only as the checker (or as the timed CPU restatement of the reference).

Every function cites the reference file:line it restates.  The reference's
Fortran cannot be compiled in this container (no Fortran compiler, no MKL), so
the restatement is pinned against the reference's own known-answer programs
and validation records instead:

* ``app/half_energy_check.F90:19-34``  occupation known answers;
* ``app/half_energy_check.F90:58-97``  the explicit 3-plane-wave, 2-projector
  non-local force vs its central finite difference (tolerance 2e-9);
* ``app/half_force_check.F90:139-153`` dD/dR vs central difference at fixed
  Veff (tolerance 2e-4);
* ``docs/validation/si_gamma_basis.json`` / ``half_vs_happy_si_slice.json``
  (Si primitive cell, 400 eV, Gamma: 725 plane waves, kinetic checksum
  172858.94956152519 eV) and ``si_arbitrary_kpoint.json`` (733 plane waves at
  k = [0.125, 0.25, 0.375]).

Those pins are checked in ``tests/test_oracle_pins.py``.
"""
