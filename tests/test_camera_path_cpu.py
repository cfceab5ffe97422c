"""Camera-path text format and replay semantics of the reference scene (Scene.cpp:2343-2366 loader,
2403-2421 recordStep, 2424-2479 replayStep / shouldFreeze / shouldAccumulate, 1567-1575 update)."""
import pytest


def test_record_format_and_round_trip(rs, tmp_path):
    import reservoir_splatting_b200.camera_path as CP
    frames = [((1.5, 2.0, -3.25), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0)), ((1e-05, 123456.7, -0.1), (2.0, 3.0, 4.0), (0.0, 0.0, 1.0))]
    p = tmp_path / "path.txt"
    CP.write_camera_path(p, frames)
    # std::ostream defaults: six significant digits, a blank line after each frame
    assert p.read_text() == "1.5 2 -3.25\n0 1 0\n0 1 0\n\n1e-05 123457 -0.1\n2 3 4\n0 0 1\n\n"
    back = CP.read_camera_path(p)
    assert back[0] == frames[0]
    assert back[1] == ((1e-05, 123457.0, -0.1), (2.0, 3.0, 4.0), (0.0, 0.0, 1.0))


def test_loader_reads_triples_and_drops_an_incomplete_frame(rs, tmp_path):
    import reservoir_splatting_b200.camera_path as CP
    p = tmp_path / "path.txt"
    p.write_text("0 0 5\n0 0 0\n0 1 0\n\n1 0 5\n1 0 0\n0 1 0\n2 0 5\n")
    assert CP.read_camera_path(p) == [((0, 0, 5), (0, 0, 0), (0, 1, 0)), ((1, 0, 5), (1, 0, 0), (0, 1, 0))]


def _frames(n):
    return [((float(i), 0.0, 5.0), (float(i), 0.0, 0.0), (0.0, 1.0, 0.0)) for i in range(n)]


def test_replay_loops_and_resets_on_the_first_frame(rs):
    import reservoir_splatting_b200.camera_path as CP
    r = CP.CameraPathReplayer(_frames(3))
    steps = [r.update() for _ in range(7)]
    assert [s.frame for s in steps] == [0, 1, 2, 0, 1, 2, 0]
    assert [s.should_reset for s in steps] == [True, False, False, True, False, False, True]
    assert not any(s.frozen for s in steps)
    assert steps[1].position == (1.0, 0.0, 5.0)


def test_freeze_frame_holds_until_unfrozen(rs):
    import reservoir_splatting_b200.camera_path as CP
    r = CP.CameraPathReplayer(_frames(4), freeze_frame_id=2)
    steps = [r.update() for _ in range(5)]
    assert [s.frame for s in steps] == [0, 1, 2, 2, 2]
    assert [s.frozen for s in steps] == [False, False, True, True, True]
    r.unfreeze()
    assert [(s.frame, s.frozen) for s in (r.update(), r.update(), r.update())] == [(3, False), (0, False), (1, False)]


def test_replay_for_accumulation_never_freezes(rs):
    import reservoir_splatting_b200.camera_path as CP
    r = CP.CameraPathReplayer(_frames(4), freeze_frame_id=1, replay_accumulation=True)
    steps = [r.update() for _ in range(8)]
    assert [s.frame for s in steps] == [0, 1, 2, 3, 0, 1, 2, 3]
    assert not any(s.frozen for s in steps)
    assert [s.accumulate for s in steps] == [False, True, False, False, False, True, False, False]


def test_empty_path_is_rejected(rs):
    import reservoir_splatting_b200.camera_path as CP
    with pytest.raises(ValueError):
        CP.CameraPathReplayer([])
