"""discoeb_b200: the per-k-mode linear perturbation solve of DISCO-EB on sm_100a.

Host-side mirror of the reference package ``discoeb`` for this path:
``background.evolve_background``, ``perturbations.evolve_perturbations``,
``perturbations.evolve_perturbations_batched``, ``perturbations.get_power`` and
``perturbations.compute_time_derivatives``; the solve itself runs in
``libdiscoeb_b200.so`` (C ABI in include/discoeb.h).
"""
__version__ = "0.1.0"
