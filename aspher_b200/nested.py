"""solve_nested for the fft / periodic backends (filled in by the nested driver)."""


def solve_nested(*args, **kwargs):
    raise NotImplementedError("solve_nested is not built yet")
