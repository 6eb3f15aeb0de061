"""Namespace with the submodule layout of the reference's ``libculoki``
(and the host-side ``libloki`` configs/plans), so code written against the
reference reads the same:

    libculoki.configs.PulsarSearchConfig
    libculoki.plans.{FFAPlanTime, FFARegionPlannerTime, generate_ffa_regions}
    libculoki.ffa.{FFACUDA, FFAFreqSweepCUDA, compute_ffa_time_cuda, compute_ffa_scores_cuda}
    libculoki.fold.compute_brute_fold_time_cuda
    libculoki.scores.{snr_boxcar_3d, snr_boxcar_3d_max, snr_boxcar_2d_max,
                      generate_box_width_trials}
    libculoki.prune.{EPMultiPassCUDA, PruneCUDA}
"""

from . import configs, ffa, fold, plans, prune, scores  # noqa: F401
