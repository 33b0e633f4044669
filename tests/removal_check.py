"""Checks of removal records (aero_info) that hold for any correct mc_coag:
every particle ID present before a step, plus every ID the step handed out,
ends up either among the particles after the step or in exactly one
removal record, never both; a record's other_id (the particle a coagulation
produced, or the target of a per-particle coagulation) is 0 for
AERO_INFO_COAG removals that created nothing and otherwise names a particle
that exists after the step or was itself removed later in it."""
import numpy as np

INFO_COAG, INFO_HALVED, INFO_WEIGHT = 2, 3, 4


def check_id_accounting(ids_before, next_id_before, next_id_after, ids_after, rec):
    new = np.arange(next_id_before, next_id_after, dtype=np.int64)
    before = np.concatenate([np.asarray(ids_before, np.int64), new])
    after = np.asarray(ids_after, np.int64)
    removed = np.asarray(rec["id"], np.int64)
    assert len(np.unique(removed)) == len(removed), "an ID removed twice"
    assert len(np.intersect1d(removed, after)) == 0, "a removed ID is still present"
    # every removed ID existed; every ID that existed, or was handed out in
    # the step, is now present or removed
    assert np.isin(removed, before).all(), "a record names an ID that never existed"
    accounted = np.union1d(after, removed)
    missing = np.setdiff1d(before, accounted)
    assert len(missing) == 0, f"{len(missing)} particles vanished without a record"
    assert np.isin(after, before).all(), "a particle with an ID from nowhere"
    other = np.asarray(rec["other_id"], np.int64)
    nz = other != 0
    assert np.isin(other[nz], np.union1d(after, removed)).all(), "other_id names no particle"
    assert np.isin(np.asarray(rec["action"]), [INFO_COAG, INFO_HALVED, INFO_WEIGHT]).all()
