"""The module paths of gbasis's integrals that this engine replaces, so that switching is a
change of import prefix: ``gbasis.integrals.electron_repulsion`` becomes
``gbasis_b200.integrals.electron_repulsion``, and likewise for ``_schwarz_screening``,
``point_charge`` and ``nuclear_electron_attraction``.  Each module re-exports the engine's
functions and classes under the reference's names."""
