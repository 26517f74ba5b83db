"""Calculator base with the ``results`` dict and ``calculate`` contract."""
all_changes = ["positions", "numbers", "cell", "pbc"]


class Calculator:
    def __init__(self, **kwargs):
        self.results = {}
        self.atoms = None

    def calculate(self, atoms=None, properties=None, system_changes=all_changes):
        if atoms is not None:
            self.atoms = atoms
        self.results = {}
