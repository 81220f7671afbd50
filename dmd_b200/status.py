"""Progress table and ns/day (python/dmd/status.py:4-51)."""
import time


class SimulationStatus:
    """Tracks and prints simulation progress (GROMACS-style)."""

    def __init__(self, engine, dt: float = 0.002, interval: int = 100):
        self.engine = engine
        self.dt = dt
        self.interval = interval
        self.t0 = time.time()
        self.step0 = 0

    def start(self):
        self.t0 = time.time()
        self.step0 = self.engine.current_step
        cols = f"{'Step':>10} {'Time (ps)':>10} {'PE (kJ/mol)':>14} {'Box (nm)':>10} {'ns/day':>8}"
        print(cols)
        print("-" * len(cols))

    def step(self):
        step = self.engine.current_step
        if step % self.interval == 0:
            elapsed = time.time() - self.t0
            ns_day = _ns_per_day(step - self.step0, elapsed, self.dt)
            print(f"{step:>10} {self.engine.current_time:>10.4f} "
                  f"{self.engine.potential_energy:>14.4f} {self.engine.box_size:>10.4f} "
                  f"{ns_day:>8.1f}")

    def finish(self):
        elapsed = time.time() - self.t0
        steps = self.engine.current_step - self.step0
        print(f"\r  [{steps} steps in {elapsed:.1f}s]  ns/day={_ns_per_day(steps, elapsed, self.dt):.1f}")
        print()


def _ns_per_day(steps: int, elapsed_s: float, dt_ps: float) -> float:
    if elapsed_s <= 0 or steps <= 0:
        return 0.0
    return dt_ps * steps / elapsed_s * 86.4
