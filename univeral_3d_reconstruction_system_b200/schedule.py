"""Full training schedules with a PSNR trajectory (host orchestration over the C ABI).

A schedule run trains a Trainer to the end of its schedule in chunks; after every chunk it reads
the device time of the chunk (CUDA events on the trainer's stream) and evaluates the mean training-view
PSNR (Trainer::evaluatePsnr, Trainer.cpp:180-192), which is not counted as training time. From the
trajectory, time-to-PSNR is the training time at which the PSNR first reaches a target, interpolated
linearly inside the chunk that crosses it.
"""
from __future__ import annotations

from dataclasses import dataclass, field

from . import api


@dataclass
class ScheduleResult:
    iterations: list = field(default_factory=list)  # iteration after each chunk
    seconds: list = field(default_factory=list)     # cumulative device training time (s)
    psnr: list = field(default_factory=list)        # evaluatePsnr after each chunk
    gaussians: list = field(default_factory=list)
    initial_psnr: float = 0.0

    @property
    def final_psnr(self) -> float:
        return self.psnr[-1] if self.psnr else self.initial_psnr

    @property
    def total_seconds(self) -> float:
        return self.seconds[-1] if self.seconds else 0.0

    def time_to_psnr(self, target: float) -> float | None:
        """Training seconds until the PSNR first reaches `target` (None if never)."""
        prev_t, prev_p = 0.0, self.initial_psnr
        if prev_p >= target:
            return 0.0
        for t, p in zip(self.seconds, self.psnr):
            if p >= target:
                f = (target - prev_p) / max(p - prev_p, 1e-12)
                return prev_t + f * (t - prev_t)
            prev_t, prev_p = t, p
        return None

    def as_dict(self) -> dict:
        return {"iterations": self.iterations, "seconds": [round(s, 5) for s in self.seconds],
                "psnr": [round(p, 4) for p in self.psnr], "gaussians": self.gaussians,
                "initial_psnr": round(self.initial_psnr, 4), "final_psnr": round(self.final_psnr, 4),
                "train_seconds": round(self.total_seconds, 4)}


def run_schedule(trainer: api.Trainer, total_iterations: int, chunk: int = 500,
                 evaluate: bool = True) -> ScheduleResult:
    res = ScheduleResult()
    res.initial_psnr = trainer.evaluatePsnr() if evaluate else 0.0
    elapsed = 0.0
    it = trainer.iteration()
    while it < total_iterations and not trainer.done():
        k = min(chunk, total_iterations - it)
        elapsed += trainer.time_steps(k) * 1e-3
        it = trainer.iteration()
        res.iterations.append(it)
        res.seconds.append(elapsed)
        res.gaussians.append(trainer.size())
        res.psnr.append(trainer.evaluatePsnr() if evaluate else 0.0)
    return res
