"""Camera-path record and replay in the reference's text format, with its freeze-frame semantics.

The reference records the camera of every frame to a text file and replays it in a loop
(Falcor Scene.cpp: recordStep :2403-2421, the loader of the "Load User Input File" button
:2343-2366, replayStep :2424-2440, shouldFreeze / shouldAccumulate :2462-2479; README.md:66-72):

* a frame is three lines ``x y z`` -- position, target, up -- written with the C++ stream's default
  float format (six significant digits) and followed by an empty line;
* replay starts the temporal history afresh on the first frame of every loop (the scene's reset
  flag); with a freeze frame id >= 0 the scene freezes (rs_freeze: the previous frame's history is
  kept) when that frame is applied and stays on it until unfrozen, unless the sequence is replayed
  for accumulation, where that frame is the one that accumulates instead.
"""
from __future__ import annotations

import dataclasses
from pathlib import Path


def _fmt(x: float) -> str:
    # std::ostream << float: %g with precision 6
    return format(float(x), "g")


class CameraPathRecorder:
    """Appends one frame per `record` call to a text file (Scene::recordStep)."""

    def __init__(self, path):
        self.path = Path(path)
        self._f = open(self.path, "w")
        self.frames = 0

    def record(self, position, target, up):
        for v in (position, target, up):
            self._f.write(" ".join(_fmt(c) for c in v) + "\n")
        self._f.write("\n")
        self.frames += 1

    def record_camera(self, camera):
        self.record(camera.position, camera.target, camera.up)

    def close(self):
        if self._f:
            self._f.close()
            self._f = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def read_camera_path(path) -> list[tuple[tuple, tuple, tuple]]:
    """(position, target, up) of every complete frame: whitespace-separated floats read in triples,
    as the reference's loader does; a trailing incomplete frame is dropped."""
    vals = []
    for tok in Path(path).read_text().split():
        try:
            vals.append(float(tok))
        except ValueError:
            break
    frames = []
    for i in range(0, len(vals) - len(vals) % 9, 9):
        v = vals[i:i + 9]
        frames.append((tuple(v[0:3]), tuple(v[3:6]), tuple(v[6:9])))
    return frames


def write_camera_path(path, frames):
    with CameraPathRecorder(path) as r:
        for pos, tgt, up in frames:
            r.record(pos, tgt, up)


@dataclasses.dataclass
class ReplayStep:
    frame: int          # index in the sequence of the camera to render with
    position: tuple
    target: tuple
    up: tuple
    should_reset: bool  # start the temporal history afresh (set on the first frame of a loop)
    frozen: bool        # the scene is frozen for this frame (rs_freeze: the previous history is kept)
    accumulate: bool    # the frame that accumulates (replay for accumulation)


class CameraPathReplayer:
    """Loops over a recorded path (Scene::updateSelectedCamera :1567-1575 with replayStep).

    Each `update` is the scene update before a frame: while the scene is not frozen it applies the
    next camera of the loop, sets the reset flag (first frame of the loop) and freezes the scene when
    the applied frame is `freeze_frame_id`; while frozen it changes nothing, so the same camera and
    flags are rendered again, until `unfreeze`.  `replay_accumulation` never freezes and instead
    marks that frame as the one to accumulate.  freeze_frame_id = -1 never freezes."""

    def __init__(self, frames, freeze_frame_id: int = -1, replay_accumulation: bool = False):
        if not frames:
            raise ValueError("empty camera path")
        self.frames = list(frames)
        self.freeze_frame_id = int(freeze_frame_id)
        self.replay_accumulation = bool(replay_accumulation)
        self.count = 0           # mRecordedFrameCount: the next frame to apply
        self.current = None      # the frame applied last
        self.should_reset = False
        self.frozen = False

    @classmethod
    def load(cls, path, **kw):
        return cls(read_camera_path(path), **kw)

    def _last(self) -> int:
        n = len(self.frames)
        return (self.count - 1 + n) % n

    def update(self) -> ReplayStep:
        if not self.frozen:
            frame = self.count
            self.should_reset = frame == 0
            self.current = frame
            self.count = (self.count + 1) % len(self.frames)
            self.frozen = (not self.replay_accumulation) and self._last() == self.freeze_frame_id
        pos, tgt, up = self.frames[self.current]
        return ReplayStep(self.current, pos, tgt, up, self.should_reset, self.frozen, self._last() == self.freeze_frame_id)

    def unfreeze(self):
        self.frozen = False

    def reset(self):
        """Scene::resetReplayer: the next update applies frame 0."""
        self.count = 0

    def camera(self, step: ReplayStep, template):
        """`template` (a scenes.Camera) with the step's position, target and up."""
        return dataclasses.replace(template, position=tuple(step.position), target=tuple(step.target), up=tuple(step.up))


def replay_frame(pass_, replayer: CameraPathReplayer, template, **execute_kw) -> ReplayStep:
    """One frame of `pass_` (a ReservoirSplatting) along the path: the scene update, then the frame
    rendered with the step's camera, reset flag and freeze state."""
    step = replayer.update()
    pass_.freeze(step.frozen)
    pass_.execute(replayer.camera(step, template), should_reset=step.should_reset, **execute_kw)
    return step
