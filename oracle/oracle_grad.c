/* gradient restatement: filled in below */
