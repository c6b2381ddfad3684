"""Stand-in for prettytable (only imported by Bolt's timing table printer)."""


class PrettyTable(object):
    def __init__(self, *args, **kw):
        self.rows = []

    def add_row(self, row):
        self.rows.append(row)

    def __str__(self):
        return '\n'.join(str(r) for r in self.rows)
