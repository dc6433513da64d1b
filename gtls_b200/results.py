"""Result record of a search (the reference's ``src/gputls/results.py:1-24``)."""


class gtlsResult(object):
    """The results of a GTLS search: same attribute names as the reference."""

    def __init__(self, periods, period, rawDuration, durationPoints, rawDurations, duration, depth, T0, SDE,
                 chi2, transitTimes, power, snr, snrPink, snrFit, snrFitPink, raw_power, raw_chi2,
                 possiblePeriodsIndices, possiblePeriods, diagnostics=None):
        self.periods = periods
        self.period = period
        self.rawDuration = rawDuration
        self.durationPoints = durationPoints
        self.rawDurations = rawDurations
        self.duration = duration
        self.depth = depth
        self.T0 = T0
        self.SDE = SDE
        self.chi2 = chi2
        self.transitTimes = transitTimes
        self.power = power
        self.snr = snr
        self.snrPink = snrPink
        self.snrFit = snrFit
        self.snrFitPink = snrFitPink
        self.raw_power = raw_power
        self.raw_chi2 = raw_chi2
        self.possiblePeriodsIndices = possiblePeriodsIndices
        self.possiblePeriods = possiblePeriods
        # implementation details of this run (batch size, precision, argmin location, ...)
        self.diagnostics = diagnostics or {}
